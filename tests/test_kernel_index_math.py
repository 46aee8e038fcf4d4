"""Index arithmetic the CUDA kernels rely on, restated in numpy and checked
exhaustively on the CPU:

* the strict-upper-triangle enumeration of same-species triplet blocks
  (fill_chunks in csrc/cuda/mb_kernels.cu, the candidate loop of atom_pass
  in csrc/cuda/mb_batch.cu): candidate c -> (row, col) from one FP32 square
  root, corrected by one row either way;
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
