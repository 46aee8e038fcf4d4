"""Index arithmetic the CUDA kernels rely on, restated in numpy and checked
exhaustively on the CPU:

* the strict-upper-triangle enumeration of same-species triplet blocks
  (fill_chunks in csrc/cuda/mb_kernels.cu, the candidate loop of atom_pass
  in csrc/cuda/mb_batch.cu): candidate c -> (row, col) from one FP32 square
  root, corrected by one row either way;
* the per-lane (row, position) cursor of k_trip's candidate pairs
  (csrc/cuda/mb_kernels.cu): lane l visits candidates l, l + 32, ... of a
  triangular or rectangular species block, advancing the cursor by 32;
* the tensor-core staging slots of k_efs / k_efs_leg (stg_slot) and the
  48-byte neighbour rows of k_efs_leg: a bijection onto the warp's rows,
  and bank-conflict-free for the accesses the kernels make (32 banks of 4
  bytes; an access of w bytes a lane served 128 / w lanes at a time);
* the segmented warp sum of the reverse passes (leg_run_conv in
  csrc/cuda/mb_kernels.cu, the reverse triplet stage of
  csrc/cuda/mb_batch.cu): with equal keys contiguous within a round, the
  first lane of each run ends with the run's total;
* the lane layouts of the recursive-halving warp reductions
  (warp_reduce64f: lane l ends with cells 2l and 2l+1; warp_reduce16f:
  lanes l and l^1 end with cell (l >> 1) & 15)."""
from __future__ import annotations

import numpy as np
import pytest

F32 = np.float32


def _tri_rows_cols(na, sqrt_ulps=0):
    """The kernels' mapping, in FP32 as the device computes it, with the
    square root moved by `sqrt_ulps` units in the last place."""
    c = np.arange(na * (na - 1) // 2, dtype=np.int64)
    tb = F32(2 * na - 1)
    s = np.sqrt((tb * tb - F32(8) * c.astype(F32)).astype(F32)).astype(F32)
    for _ in range(abs(sqrt_ulps)):
        s = np.nextafter(s, F32(np.inf) if sqrt_ulps > 0 else F32(-np.inf))
    r = np.trunc((F32(0.5) * (tb - s)).astype(F32)).astype(np.int64)
    r = np.where((r + 1) * (2 * na - r - 2) // 2 <= c, r + 1, r)
    r = np.where(r * (2 * na - r - 1) // 2 > c, r - 1, r)
    r = np.clip(r, 0, na - 2)
    col = np.clip(c - r * (2 * na - r - 1) // 2 + r + 1, r + 1, na - 1)
    return r, col


@pytest.mark.parametrize("ulps", [-2, -1, 0, 1, 2])
def test_triangle_enumeration_is_row_major_and_exact(ulps):
    """Every block size the kernels enumerate as a triangle (the batched
    kernel's 96-neighbour capacity; k_efs up to 256 neighbours of a species)
    gives exactly the row-major strict upper triangle, even with the square
    root off by two units in the last place."""
    sizes = list(range(2, 97)) + [128, 160, 200, 255, 256]
    for na in sizes:
        r, col = _tri_rows_cols(na, ulps)
        rr, cc = np.triu_indices(na, 1)
        np.testing.assert_array_equal(r, rr, err_msg=f"rows, na={na}")
        np.testing.assert_array_equal(col, cc, err_msg=f"cols, na={na}")


def _halving(v, steps):
    """Recursive halving across 32 lanes: at step k (offset 16 >> k) a lane
    keeps one half of its cells (the upper half if its offset bit is set)
    and adds its partner's copy of that half."""
    v = v.copy()
    lanes = np.arange(32)
    for step in range(steps):
        off, half = 16 >> step, v.shape[1] // 2
        upper = (lanes & off) != 0
        partner = lanes ^ off
        keep = np.where(upper[:, None], v[:, half:], v[:, :half])
        send = np.where(upper[:, None], v[:, :half], v[:, half:])
        v = keep + send[partner]
    return v


def test_warp_reduce64_lane_layout():
    rng = np.random.default_rng(0)
    v = rng.normal(size=(32, 64))
    out = _halving(v, 5)
    tot = v.sum(0)
    lanes = np.arange(32)
    np.testing.assert_allclose(out[:, 0], tot[2 * lanes], rtol=1e-12)
    np.testing.assert_allclose(out[:, 1], tot[2 * lanes + 1], rtol=1e-12)


def test_warp_reduce16_lane_layout():
    rng = np.random.default_rng(1)
    v = rng.normal(size=(32, 16))
    out = _halving(v, 4)[:, 0]
    lanes = np.arange(32)
    done = out + out[lanes ^ 1]
    np.testing.assert_allclose(done, v.sum(0)[(lanes >> 1) & 15], rtol=1e-12)


def _cursor_walk(na, nb, tri, lane):
    """k_trip's cursor for one lane, restated: the (candidate, row, column)
    it visits, checking on the way that every index it would use lies in
    the block."""
    C = na * (na - 1) // 2 if tri else na * nb
    out = []
    if C <= 0:
        return out
    rmax = na - 2 if tri else na - 1

    def length(r):
        return na - 1 - r if tri else nb

    r, p = 0, lane
    while p >= length(r) and r < rmax:
        p -= length(r)
        r += 1
    c = lane
    while c < C:
        col = r + 1 + p if tri else p
        assert 0 <= r <= rmax
        assert (r + 1 <= col <= na - 1) if tri else (0 <= col <= nb - 1)
        out.append((c, r, col))
        c += 32
        p += 32
        while p >= length(r) and r < rmax:
            p -= length(r)
            r += 1
    return out


@pytest.mark.parametrize("tri", [True, False])
def test_triplet_cursor_matches_row_major_order(tri):
    """For every block shape up to the leg path's 128-entry capacity (all
    triangles; rectangles up to 128 x 64 and a sample beyond), each lane's
    cursor visits exactly the row-major candidates c = lane + 32 k, and
    every row and column it produces lies inside the block."""
    sizes = [(na, na) for na in range(0, 129)] if tri else \
        [(na, nb) for na in range(0, 129) for nb in range(0, 65)] + [(na, nb) for na in (1, 7, 64, 128) for nb in
                                                                    (65, 97, 128)]
    for na, nb in sizes:
        C = na * (na - 1) // 2 if tri else na * nb
        if C <= 0:
            continue
        if tri:
            r_ref, c_ref = _tri_rows_cols(na)
        else:
            cc = np.arange(C)
            r_ref, c_ref = cc // nb, cc % nb
        for lane in range(32):
            walk = _cursor_walk(na, nb, tri, lane)
            assert [w[0] for w in walk] == list(range(lane, C, 32))
            for c, r, col in walk:
                assert r == r_ref[c] and col == c_ref[c], (na, nb, lane, c)


def _stg_slot(t, q):
    """stg_slot in csrc/cuda/mb_kernels.cu (rows of 16 doubles)."""
    return t * 16 + ((q + 4 * (t & 3) + ((t >> 2) & 3)) & 15)


def _wavefronts(byte_addrs, width):
    """Shared-memory wavefronts of one warp access of `width` bytes a lane:
    lanes are served 128 / width at a time; within a phase, distinct 4-byte
    words in one bank serialise (one word read by several lanes is one)."""
    per = 128 // width
    total = 0
    for p in range(0, 32, per):
        banks = {}
        for a in byte_addrs[p:p + per]:
            for k in range(width // 4):
                word = a // 4 + k
                banks.setdefault(word % 32, set()).add(word)
        total += max(len(v) for v in banks.values())
    return total


def test_staging_slots_are_a_conflict_free_bijection():
    slots = {_stg_slot(t, q) for t in range(32) for q in range(16)}
    assert slots == set(range(32 * 16))
    # the writes: every lane its own triplet t = lane, one value q at a time
    for q in range(16):
        assert _wavefronts([8 * _stg_slot(lane, q) for lane in range(32)], 8) == 2
    # the mma operand reads: step st takes triplets 4 st + (lane & 3), value (lane >> 2) (+ 8)
    for st in range(8):
        for off in (0, 8):
            assert _wavefronts([8 * _stg_slot(4 * st + (l & 3), off + (l >> 2)) for l in range(32)], 8) == 2


def test_neighbour_rows_are_conflict_free_for_consecutive_entries():
    """k_efs_leg's rows {x, y, z, 1/r, r, 0} (48 bytes) read as two 16-byte
    loads: consecutive entries, as a round of consecutive list entries
    gives the b side, take the minimum 4 wavefronts a load; a 32-byte row
    would take 8."""
    for base in range(0, 64):
        for h in range(2):
            assert _wavefronts([48 * (base + b) + 16 * h for b in range(32)], 16) == 4
    assert _wavefronts([32 * b for b in range(32)], 16) == 8


def _segmented_sum(keys, vals):
    """The kernels' doubling steps: lane l adds lane l + o's partial when
    both hold the same key (o = 1, 2, 4, 8, 16; shfl_down leaves lanes past
    31 their own value)."""
    v = np.array(vals, dtype=np.float64)
    k = list(keys)
    for o in (1, 2, 4, 8, 16):
        nv = v.copy()
        for l in range(32):
            if l + o < 32 and k[l + o] == k[l]:
                nv[l] = v[l] + v[l + o]
        v = nv
    return v


def test_segmented_warp_sum_heads_hold_their_run_totals():
    rng = np.random.default_rng(3)
    for _ in range(2000):
        # a round of a row-major list: nondecreasing keys, idle lanes at the
        # end carry keys of their own (the kernels use 256 + lane / -1 - lane)
        n = int(rng.integers(1, 33))
        keys = sorted(rng.integers(0, int(rng.integers(1, 12)), n).tolist()) + [1000 + l for l in range(32 - n)]
        vals = rng.normal(size=32)
        out = _segmented_sum(keys, vals)
        for l in range(32):
            if l == 0 or keys[l - 1] != keys[l]:  # the run's first lane adds it to the force
                run = [m for m in range(l, 32) if keys[m] == keys[l]]
                assert run == list(range(l, l + len(run)))
                assert abs(out[l] - sum(vals[m] for m in run)) < 1e-12
    # the order matters: a key split by another one would be counted twice
    keys = [0, 1, 0] + [100 + l for l in range(29)]
    out = _segmented_sum(keys, np.ones(32))
    assert out[0] + out[2] != 2.0
