/*
 * mb_kernels.cu -- sm_100a kernels of libmaise_b200 (FP64 one-structure path).
 *
 *   k_wrap          wrap positions into the cell (JAR, src/cell.c:445-508)
 *   k_nlist_brute   all (atom, image) pairs within Rc (LIST, src/cell.c:82-185)
 *   k_cell_*        integer cell-list build (bin, count, scan, fill) and
 *   k_nlist_cell    the same neighbour set from the 27 adjacent cells
 *   k_efs           one CTA per central atom: G2/G4 descriptors
 *                   (src/nprs.c:500-566), MLP forward and dE/dG
 *                   (src/nmlp.c:367-431), then the reverse pass that turns
 *                   dE_i/dG_i into forces on i and its neighbours and the
 *                   virial (src/nprs.c:567-770 contracted as in
 *                   src/nmlp.c:433-479) without materialising dG/dx
 *   k_finalize      energy and virial reductions in fixed order, noise
 *                   zeroing and enthalpy (src/cmod.c:153-191)
 *   k_nvt_*         NVT thermostat and integrator (src/cmod.c:403-453)
 *
 * The wrap and the neighbour test use explicitly rounded operations
 * (__dadd_rn/__dmul_rn, never contracted into FMAs) in the reference's
 * operation order, so the selected neighbour set is the reference's.
 */
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>
#include <stdlib.h>

#include "../mb_internal.h"

#define FULL 0xffffffffu

namespace {

__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }

/* ------------------------------------------------------------------ */
/* wrap                                                                */
/* ------------------------------------------------------------------ */

/* JAR on atom i's position: Cartesian -> fractional, into [0, 1), back */
__device__ __forceinline__ void wrap_atom(int i, double *__restrict__ X, const mb_cell &c, int *status) {
    double x[3];
    for (int q = 0; q < 3; q++) {
        double s = 0.0;
        for (int j = 0; j < 3; j++) s = xadd(s, xmul(X[3 * i + j], c.R[3 * q + j]));
        x[q] = s;
    }
    for (int q = 0; q < 3; q++) {
        int it = 0;
        while (x[q] < 0.0 && it < 4096) { x[q] = xadd(x[q], 1.0); it++; }
        while (x[q] >= 1.0 && it < 4096) { x[q] = xsub(x[q], 1.0); it++; }
        if (!(x[q] >= 0.0 && x[q] < 1.0)) atomicOr(status, MB_ST_WRAP);
    }
    for (int q = 0; q < 3; q++) {
        double s = 0.0;
        for (int j = 0; j < 3; j++) s = xadd(s, xmul(x[j], c.L[3 * j + q]));
        X[3 * i + q] = s;
    }
}

__global__ void k_wrap(int N, double *__restrict__ X, mb_cell c, int *status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    wrap_atom(i, X, c, status);
}

/* ------------------------------------------------------------------ */
/* neighbour list                                                      */
/* ------------------------------------------------------------------ */

/* displacement of atom j's image (i0,i1,i2) from atom i and its squared
 * length, formed exactly as src/cell.c:115-121 */
__device__ __forceinline__ double image_disp(const mb_cell &c, const double *xi, const double *xj, int i0, int i1,
                                             int i2, double *d) {
    double r = 0.0;
#pragma unroll
    for (int q = 0; q < 3; q++) {
        double x = 0.0;
        x = xadd(x, xmul((double)i0, c.L[q]));
        x = xadd(x, xmul((double)i1, c.L[3 + q]));
        x = xadd(x, xmul((double)i2, c.L[6 + q]));
        x = xadd(x, xsub(xj[q], xi[q]));
        d[q] = x;
        r = xadd(r, xmul(x, x));
    }
    return r;
}

/* key of a list entry for the leg-table path: atom j and its integer image
 * (5 bits per axis, two's complement) */
__device__ __forceinline__ unsigned entry_key(int j, int i0, int i1, int i2) {
    return ((unsigned)j << 15) | (((unsigned)i0 & 31u) << 10) | (((unsigned)i1 & 31u) << 5) | ((unsigned)i2 & 31u);
}

/* one warp per atom; candidates in the reference's order (j, then images) */
__global__ void k_nlist_brute(int N, int NM, int cap, const double *__restrict__ X, mb_cell c, double rc2,
                              int *__restrict__ nn, int *__restrict__ nj, double4 *__restrict__ nd, int *status,
                              unsigned *__restrict__ nk) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= N) return;
    int i = warp;
    int w0 = 2 * c.Nq[0] + 1, w1 = 2 * c.Nq[1] + 1, w2 = 2 * c.Nq[2] + 1;
    int nimg = w0 * w1 * w2;
    long long total = (long long)N * nimg;
    double xi[3] = {X[3 * i], X[3 * i + 1], X[3 * i + 2]};
    int count = 0;
    for (long long base = 0; base < total; base += 32) {
        long long cidx = base + lane;
        bool ok = false;
        int j = 0, i0 = 0, i1 = 0, i2 = 0;
        double d[3] = {0, 0, 0}, r2 = 0.0;
        if (cidx < total) {
            j = (int)(cidx / nimg);
            int im = (int)(cidx % nimg);
            i2 = im % w2 - c.Nq[2];
            int t = im / w2;
            i1 = t % w1 - c.Nq[1];
            i0 = t / w1 - c.Nq[0];
            if (!(j == i && i0 == 0 && i1 == 0 && i2 == 0)) {
                double xj[3] = {X[3 * j], X[3 * j + 1], X[3 * j + 2]};
                r2 = image_disp(c, xi, xj, i0, i1, i2, d);
                ok = r2 < rc2;
            }
        }
        unsigned m = __ballot_sync(FULL, ok);
        int pos = count + __popc(m & ((1u << lane) - 1u));
        if (ok && pos < cap) {
            nj[(size_t)i * cap + pos] = j;
            nd[(size_t)i * cap + pos] = make_double4(d[0], d[1], d[2], sqrt(r2));
            if (nk) nk[(size_t)i * cap + pos] = entry_key(j, i0, i1, i2);
        }
        count += __popc(m);
    }
    if (lane == 0) {
        nn[i] = count < cap ? count : cap;
        if (count >= NM) atomicOr(status, MB_ST_NBR_OVERFLOW);
        if (count > cap) atomicOr(status, MB_ST_CAP_OVERFLOW);
        atomicMax(&status[1], count);
    }
}

__device__ __forceinline__ int cell_index(const mb_cell &c, const double *x, int *cq) {
    for (int q = 0; q < 3; q++) {
        double f = x[0] * c.R[3 * q] + x[1] * c.R[3 * q + 1] + x[2] * c.R[3 * q + 2];
        int k = (int)floor(f * c.M[q]);
        k = k < 0 ? 0 : (k >= c.M[q] ? c.M[q] - 1 : k);
        cq[q] = k;
    }
    return (cq[0] * c.M[1] + cq[1]) * c.M[2] + cq[2];
}

__global__ void k_cell_bin(int N, const double *__restrict__ X, mb_cell c, int *cell_of, int *cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int cq[3];
    int k = cell_index(c, X + 3 * i, cq);
    cell_of[i] = k;
    atomicAdd(&cnt[k], 1);
}

/* exclusive scan of the cell counts by one CTA of 1024 threads; start[ncell] = N */
__global__ void k_cell_scan(int ncell, const int *cnt, int *start) {
    __shared__ int wsum[32];
    const int t = threadIdx.x, nt = blockDim.x, lane = t & 31, w = t >> 5;
    const int per = (ncell + nt - 1) / nt, lo = t * per, hi = min(lo + per, ncell);
    int s = 0;
    for (int k = lo; k < hi; k++) s += cnt[k];
    int x = s; /* inclusive scan over the warp */
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        int v = lane < (nt >> 5) ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(FULL, v, o);
            if (lane >= o) v += y;
        }
        wsum[lane] = v;
    }
    __syncthreads();
    int e = x - s + (w > 0 ? wsum[w - 1] : 0);
    for (int k = lo; k < hi; k++) {
        start[k] = e;
        e += cnt[k];
    }
    if (t == nt - 1) start[ncell] = e;
}

__global__ void k_cell_fill(int N, const int *cell_of, const int *start, int *cursor, int *atoms) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int k = cell_of[i];
    int pos = atomicAdd(&cursor[k], 1);
    atoms[start[k] + pos] = i;
}

/* order each cell's atoms by index so the neighbour order is deterministic:
 * one warp per cell, each atom placed at its rank (the number of smaller
 * indices in the cell; indices are distinct); cells of more than
 * 32 * CELL_SORT_PER_LANE atoms are sorted by one lane */
#define CELL_SORT_PER_LANE 8
__global__ void k_cell_sort(int ncell, const int *start, int *atoms) {
    const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (k >= ncell) return;
    const int lo = start[k], n = start[k + 1] - lo;
    if (n <= 32 * CELL_SORT_PER_LANE) {
        int v[CELL_SORT_PER_LANE], r[CELL_SORT_PER_LANE];
#pragma unroll
        for (int q = 0; q < CELL_SORT_PER_LANE; q++) {
            const int e = q * 32 + lane;
            v[q] = e < n ? atoms[lo + e] : 0x7fffffff;
            r[q] = 0;
        }
        const int rounds = (n + 31) >> 5;
        for (int f = 0; f < n; f++) {
            const int w = atoms[lo + f];
#pragma unroll
            for (int q = 0; q < CELL_SORT_PER_LANE; q++)
                if (q < rounds) r[q] += w < v[q];
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < CELL_SORT_PER_LANE; q++)
            if (q * 32 + lane < n) atoms[lo + r[q]] = v[q];
    } else if (lane == 0) {
        for (int a = lo + 1; a < lo + n; a++) {
            int v = atoms[a], b = a - 1;
            while (b >= lo && atoms[b] > v) {
                atoms[b + 1] = atoms[b];
                b--;
            }
            atoms[b + 1] = v;
        }
    }
}

/* One warp per atom over the 27 adjacent cells.  Periodic directions have
 * at least 3 bins no thinner than Rc, so every image within Rc lies in an
 * adjacent bin and each (atom, image) pair is visited once; the exact test
 * then selects the reference's set.  The 27 cells' atom ranges are laid end
 * to end (cell order a, b, e; atoms in index order within a cell) and
 * walked 32 candidates per round, every lane busy. */
__global__ void k_nlist_cell(int N, int NM, int cap, const double *__restrict__ X, mb_cell c, double rc2,
                             const int *__restrict__ cell_of, const int *__restrict__ start,
                             const int *__restrict__ atoms, int *__restrict__ nn, int *__restrict__ nj,
                             double4 *__restrict__ nd, int *status, unsigned *__restrict__ nk) {
    __shared__ int s_off[4][32], s_lo[4][32], s_img[4][32];
    const int w = (threadIdx.x >> 5) & 3;
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= N) return;
    int i = warp;
    double xi[3] = {X[3 * i], X[3 * i + 1], X[3 * i + 2]};
    int ci = cell_of[i];
    int cq[3] = {ci / (c.M[1] * c.M[2]), (ci / c.M[2]) % c.M[1], ci % c.M[2]};
    /* lane k < 27 describes adjacent cell k = 9 (a+1) + 3 (b+1) + (e+1) */
    int lo = 0, cnt = 0, pimg = 0;
    if (lane < 27) {
        const int dd[3] = {lane / 9 - 1, (lane / 3) % 3 - 1, lane % 3 - 1};
        int cc[3], img[3];
        bool skip = false;
        for (int q = 0; q < 3; q++) {
            int k = cq[q] + dd[q];
            img[q] = 0;
            if (q < c.ND) {
                if (k < 0) { k += c.M[q]; img[q] = -1; }
                else if (k >= c.M[q]) { k -= c.M[q]; img[q] = 1; }
            } else if (k < 0 || k >= c.M[q]) {
                skip = true;
            }
            cc[q] = k;
        }
        if (!skip) {
            const int cell = (cc[0] * c.M[1] + cc[1]) * c.M[2] + cc[2];
            lo = start[cell];
            cnt = start[cell + 1] - lo;
        }
        pimg = (img[0] + 1) * 9 + (img[1] + 1) * 3 + (img[2] + 1);
    }
    int off = cnt; /* inclusive scan of the cell sizes */
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, off, o);
        if (lane >= o) off += y;
    }
    const int total = __shfl_sync(FULL, off, 31);
    s_off[w][lane] = off - cnt; /* exclusive */
    s_lo[w][lane] = lo;
    s_img[w][lane] = pimg;
    __syncwarp();
    int count = 0;
    for (int base = 0; base < total; base += 32) {
        const int t = base + lane;
        bool ok = false;
        int j = 0, img[3] = {0, 0, 0};
        double d[3] = {0, 0, 0}, r2 = 0.0;
        if (t < total) {
            /* the last of the 27 cells whose range starts at or before t */
            int k = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1)
                if (k + step < 27 && s_off[w][k + step] <= t) k += step;
            j = atoms[s_lo[w][k] + (t - s_off[w][k])];
            const int pi = s_img[w][k];
            img[0] = pi / 9 - 1;
            img[1] = (pi / 3) % 3 - 1;
            img[2] = pi % 3 - 1;
            if (!(j == i && img[0] == 0 && img[1] == 0 && img[2] == 0)) {
                double xj[3] = {X[3 * j], X[3 * j + 1], X[3 * j + 2]};
                r2 = image_disp(c, xi, xj, img[0], img[1], img[2], d);
                ok = r2 < rc2;
            }
        }
        unsigned m = __ballot_sync(FULL, ok);
        int pos = count + __popc(m & ((1u << lane) - 1u));
        if (ok && pos < cap) {
            nj[(size_t)i * cap + pos] = j;
            nd[(size_t)i * cap + pos] = make_double4(d[0], d[1], d[2], sqrt(r2));
            if (nk) nk[(size_t)i * cap + pos] = entry_key(j, img[0], img[1], img[2]);
        }
        count += __popc(m);
    }
    if (lane == 0) {
        nn[i] = count < cap ? count : cap;
        if (count >= NM) atomicOr(status, MB_ST_NBR_OVERFLOW);
        if (count > cap) atomicOr(status, MB_ST_CAP_OVERFLOW);
        atomicMax(&status[1], count);
    }
}

/* ------------------------------------------------------------------ */
/* descriptor / MLP / force kernel                                     */
/* ------------------------------------------------------------------ */

__device__ __forceinline__ double fcut(double rc, double r) { return r > rc ? 0.0 : 0.5 * (cospi(r / rc) + 1.0); }

__device__ __forceinline__ void fcut_d(double rc, double r, double &f, double &df) {
    if (r > rc) {
        f = 0.0;
        df = 0.0;
        return;
    }
    double s, co;
    sincospi(r / rc, &s, &co);
    f = 0.5 * (co + 1.0);
    df = -0.5 * CUDART_PI / rc * s;
}

/* (1 + lambda c)^zeta * 2^(1-zeta) for every (zeta, lambda), and optionally
 * the derivative in c; integer zeta by repeated squaring.  NZ and NLAM are
 * upper bounds (exact for the specialised kernels); zl = z*NLAM + l. */
/* PZ = false leaves out the normalisation powz[z] = 2^(1 - zeta) (the
 * caller folds it into the per-block grid instead: for the reference
 * bases it is a power of two, so the results are unchanged bit for bit) */
template <int NZ, int NLAM, bool PZ = true>
__device__ __forceinline__ void angular(const mb_params &P, double c, double *lz, double *lzp) {
    auto pz = [&](int z) { return PZ ? P.powz[z] : 1.0; };
    if (NZ == 4 && P.zeta_std) {
        /* zeta = 1, 2, 4, 16 (the reference bases): powers by squaring */
#pragma unroll
        for (int l = 0; l < NLAM; l++) {
            if (l >= P.nlam) break;
            const double lam = P.lam[l], b1 = 1.0 + lam * c, b2 = b1 * b1, b4 = b2 * b2, b8 = b4 * b4;
            if constexpr (PZ) {
                lz[0 * NLAM + l] = P.powz[0] * b1;
                lz[1 * NLAM + l] = P.powz[1] * b2;
                lz[2 * NLAM + l] = P.powz[2] * b4;
                lz[3 * NLAM + l] = P.powz[3] * (b8 * b8);
            } else {
                lz[0 * NLAM + l] = b1;
                lz[1 * NLAM + l] = b2;
                lz[2 * NLAM + l] = b4;
                lz[3 * NLAM + l] = b8 * b8;
            }
            if (lzp) {
                if constexpr (PZ) {
                    lzp[0 * NLAM + l] = P.powz[0] * lam;
                    lzp[1 * NLAM + l] = P.powz[1] * 2.0 * lam * b1;
                    lzp[2 * NLAM + l] = P.powz[2] * 4.0 * lam * (b2 * b1);
                    lzp[3 * NLAM + l] = P.powz[3] * 16.0 * lam * (b8 * b4 * b2 * b1);
                } else {
                    lzp[0 * NLAM + l] = lam;
                    lzp[1 * NLAM + l] = 2.0 * lam * b1;
                    lzp[2 * NLAM + l] = 4.0 * lam * (b2 * b1);
                    lzp[3 * NLAM + l] = 16.0 * lam * (b8 * b4 * b2 * b1);
                }
            }
        }
        return;
    }
#pragma unroll
    for (int l = 0; l < NLAM; l++) {
        if (l >= P.nlam) break;
        double lam = P.lam[l];
        double base = 1.0 + lam * c;
        if (P.zeta_int) {
            double sq[7];
            sq[0] = base;
#pragma unroll
            for (int k = 1; k < 7; k++) sq[k] = sq[k - 1] * sq[k - 1];
#pragma unroll
            for (int z = 0; z < NZ; z++) {
                if (z >= P.nz) break;
                int zb = P.zbits[z], mb = P.zm1bits[z];
                double pw = 1.0, pm = 1.0;
#pragma unroll
                for (int k = 0; k < 7; k++) {
                    if (zb & (1 << k)) pw *= sq[k];
                    if (mb & (1 << k)) pm *= sq[k];
                }
                lz[z * NLAM + l] = pz(z) * pw;
                if (lzp) lzp[z * NLAM + l] = pz(z) * P.zeta[z] * lam * pm;
            }
        } else {
#pragma unroll
            for (int z = 0; z < NZ; z++) {
                if (z >= P.nz) break;
                lz[z * NLAM + l] = pz(z) * pow(base, P.zeta[z]);
                if (lzp) lzp[z * NLAM + l] = pz(z) * P.zeta[z] * lam * pow(base, P.zeta[z] - 1.0);
            }
        }
    }
}

struct EfsArgs {
    int N, cap, mode;
    double urep;
    const int *nn, *nj;
    const double4 *nd;
    const int *spc;
    const mb_params *params;
    const double *weights;
    double *EA, *EU, *G, *F, *vir;
    unsigned long long *counters; /* [0] pairs, [1] accepted forward triplets */
    size_t smem_group;            /* shared-memory bytes of one atom group */
    int tl_cap;                   /* triplet-list entries of one atom group */
};

/* shared-memory carve-up of one atom group of k_efs */
struct EfsSmem {
    int *j, *sp;
    double4 *d;
    double *ir, *fa, *fb, *P, *Fnb, *G, *grid, *red, *tmp, *h;
    double *stage; /* per warp: 32 triplets x EFS_STG doubles (tensor-core forward) */
    unsigned *tl;  /* accepted (j,k) pairs: per-warp regions of tlw entries */
    int *blk;      /* [block][warp][2] ranges of each warp's region per species block */
    int *seg;      /* [0..3] counts, [4..7] offsets */
};

#define MB_MAX_BLOCKS 6 /* species blocks (a<=b) for 3 species */

__host__ __device__ inline size_t align8(size_t x) { return (x + 7) & ~(size_t)7; }
__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }
/* row stride of the per-neighbour exponential factors: even, so that rows
 * start on 16 bytes (the neighbour capacity is a multiple of 8) */
__host__ __device__ constexpr int nep(int ne) { return (ne + 1) & ~1; }

#define EFS_STG 16 /* staging row: 8 exponential + 8 angular values */

/* Staging slot of value q (0-7 exponential, 8-15 angular) of a warp's
 * triplet t (0-31): rows of 16 doubles whose columns are rotated by
 * 4 (t & 3) + ((t >> 2) & 3).  An 8-byte shared access is served a
 * half-warp at a time; the writes (one q, 16 consecutive t) and the
 * mma operand reads (4 consecutive t x 4 consecutive q) then both touch
 * 16 distinct banks.  (A padded row of 17 left the operand reads 4-way
 * conflicted.) */
__device__ __forceinline__ int stg_slot(int t, int q) { return t * EFS_STG + ((q + 4 * (t & 3) + ((t >> 2) & 3)) & 15); }

/* Sizes of the regions that share one block of memory: the forward
 * staging rows (tensor-core forward, live only while the forward triplets
 * run) and Fnb + grid + red + h (block reductions, MLP and reverse pass,
 * all after it). */
__host__ __device__ inline size_t efs_union_bytes(int cap, int nzl_cells, int warps, int stage) {
    const size_t st = stage ? sizeof(double) * warps * 32 * EFS_STG : 0;
    const size_t rest = sizeof(double) * (cap * 3 + nzl_cells + warps * 64 + 4 * MB_MAXH);
    return align16(st > rest ? st : rest);
}

__host__ __device__ inline size_t efs_smem_bytes(int cap, int D, int ne, int ng2, int nzl_cells, int warps, int tl,
                                                 int stage) {
    size_t b = 0;
    b += efs_union_bytes(cap, nzl_cells, warps, stage); /* stage | Fnb, grid, red, h */
    b += align8(sizeof(int) * cap) * 2;           /* j, sp */
    b += sizeof(double4) * cap;                   /* d */
    b += sizeof(double) * cap * 3;                /* ir, fa, fb */
    b += sizeof(double) * cap * nep(ne);          /* P */
    b += align16(sizeof(double) * D);             /* G */
    /* tmp (G2 terms) and tl (triplet list) share one region: tmp is dead
     * before the first list entry is written */
    const size_t tmp_b = sizeof(double) * cap * (ng2 > 1 ? ng2 : 1), tl_b = align8(sizeof(unsigned) * tl);
    b += tmp_b > tl_b ? tmp_b : tl_b; /* tmp | tl */
    b += align8(sizeof(int) * MB_MAX_BLOCKS * warps * 2);
    b += sizeof(int) * 8;
    return b;
}

__device__ inline EfsSmem efs_carve(char *base, int cap, int D, int ne, int ng2, int nzl_cells, int warps, int tl,
                                   int stage) {
    /* one atom group's region; `warps` = warps per atom */
    EfsSmem s;
    char *p = base;
    s.stage = (double *)p;
    s.Fnb = (double *)p;
    s.grid = s.Fnb + cap * 3;
    s.red = s.grid + nzl_cells;
    s.h = s.red + warps * 64;
    p += efs_union_bytes(cap, nzl_cells, warps, stage);
    s.d = (double4 *)p; p += sizeof(double4) * cap;
    s.ir = (double *)p; p += sizeof(double) * cap;
    s.fa = (double *)p; p += sizeof(double) * cap;
    s.fb = (double *)p; p += sizeof(double) * cap;
    s.P = (double *)p; p += sizeof(double) * cap * nep(ne);
    s.G = (double *)p; p += align16(sizeof(double) * D);
    {
        const size_t tmp_b = sizeof(double) * cap * (ng2 > 1 ? ng2 : 1), tl_b = align8(sizeof(unsigned) * tl);
        s.tmp = (double *)p;
        s.tl = (unsigned *)p;
        p += tmp_b > tl_b ? tmp_b : tl_b;
    }
    s.j = (int *)p; p += align8(sizeof(int) * cap);
    s.sp = (int *)p; p += align8(sizeof(int) * cap);
    s.blk = (int *)p; p += align8(sizeof(int) * MB_MAX_BLOCKS * warps * 2);
    s.seg = (int *)p;
    return s;
}

/* Sum of 64 per-lane values across a warp: afterwards lane l holds the
 * sums of values 2l and 2l+1 (recursive halving). */
__device__ __forceinline__ void warp_reduce64(double *v, int lane) {
#pragma unroll
    for (int step = 0; step < 5; step++) {
        const int off = 16 >> step, half = 32 >> step;
        const bool upper = (lane & off) != 0;
#pragma unroll
        for (int k = 0; k < half; k++) {
            double send = upper ? v[k] : v[k + half];
            double keep = upper ? v[k + half] : v[k];
            v[k] = keep + __shfl_xor_sync(FULL, send, off);
        }
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

template <int WPA>
__device__ __forceinline__ void group_sync() {
    if (WPA == 1)
        __syncwarp();
    else
        __syncthreads();
}

/* Reduction of a 64-cell accumulator grid over the atom's group into
 * s.red[0..63] (warp 0 adds the warps' partial sums in a fixed order). */
template <int WPA, class Smem>
__device__ __forceinline__ void group_reduce64(double *v, Smem &s, int gwarp, int lane) {
    warp_reduce64(v, lane);
    if (WPA == 1) {
        s.red[2 * lane] = v[0];
        s.red[2 * lane + 1] = v[1];
        __syncwarp();
        return;
    }
    s.red[gwarp * 64 + 2 * lane] = v[0];
    s.red[gwarp * 64 + 2 * lane + 1] = v[1];
    __syncthreads();
    if (gwarp == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < WPA; w++) {
            a += s.red[w * 64 + 2 * lane];
            b += s.red[w * 64 + 2 * lane + 1];
        }
        __syncwarp();
        s.red[2 * lane] = a;
        s.red[2 * lane + 1] = b;
    }
    __syncthreads();
}

/* As group_reduce64 for values already summed over the warp (lane l holds
 * cells 2l and 2l+1, the layout of a tensor-core accumulator fragment). */
template <int WPA, class Smem>
__device__ __forceinline__ void group_store64(double v0, double v1, Smem &s, int gwarp, int lane) {
    if (WPA == 1) {
        s.red[2 * lane] = v0;
        s.red[2 * lane + 1] = v1;
        __syncwarp();
        return;
    }
    s.red[gwarp * 64 + 2 * lane] = v0;
    s.red[gwarp * 64 + 2 * lane + 1] = v1;
    __syncthreads();
    if (gwarp == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < WPA; w++) {
            a += s.red[w * 64 + 2 * lane];
            b += s.red[w * 64 + 2 * lane + 1];
        }
        __syncwarp();
        s.red[2 * lane] = a;
        s.red[2 * lane + 1] = b;
    }
    __syncthreads();
}

/* D(8x8) += A(8x4) B(4x8) in FP64 on the tensor cores (mma.sync m8n8k4):
 * lane l holds A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4) + {0, 1}]. */
__device__ __forceinline__ void dmma884(double &c0, double &c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

/* Candidates of block (a, b): the na x nb square for a != b; for a == b
 * only the strict upper triangle (col > row), enumerated directly up to 256
 * neighbours of the species (the square with the lower half skipped above) */
__device__ __forceinline__ bool block_tri(const EfsSmem &s, int a, int b) { return a == b && s.seg[a] <= 256; }
__device__ __forceinline__ int block_candidates(const EfsSmem &s, int a, int b) {
    const int na = s.seg[a], nb = s.seg[b];
    return block_tri(s, a, b) ? na * (na - 1) / 2 : na * nb;
}

/* Append the accepted candidates (j, k) of block (a, b) to this warp's
 * list region in row-major order, 32 candidates per round with every lane
 * busy, the warps of an atom taking every WPA-th round.  Square: row =
 * (c + 0.5) / nb in FP32 is exact (the fraction stays >= 0.5 / nb away from
 * an integer).  Triangle: row r starts at r (2 na - r - 1) / 2, inverted
 * with one FP32 square root and corrected by one row either way (exact for
 * na <= 256 under +-2 ulp of sqrt error).  Returns the next candidate
 * index; stops early when the region is full. */
template <int WPA, class Accept>
__device__ __forceinline__ int fill_chunks(const EfsSmem &s, int a, int b, int c, int &pos, int hi, int lane,
                                           Accept accept) {
    const int na = s.seg[a], nb = s.seg[b], oa = s.seg[4 + a], ob = s.seg[4 + b];
    const bool tri = block_tri(s, a, b);
    const int C = block_candidates(s, a, b);
    const float inv_nb = nb > 0 ? 1.0f / (float)nb : 0.0f, tb = (float)(2 * na - 1);
    for (; c < C && pos + 32 <= hi; c += 32 * WPA) {
        const int cc = c + lane;
        bool ok = false;
        int jj = 0, kk = 0;
        if (cc < C) {
            int r, col;
            if (tri) {
                r = __float2int_rz(0.5f * (tb - sqrtf(tb * tb - 8.0f * (float)cc)));
                if ((r + 1) * (2 * na - r - 2) / 2 <= cc) r++;
                else if (r * (2 * na - r - 1) / 2 > cc) r--;
                r = min(max(r, 0), na - 2);
                col = min(max(cc - r * (2 * na - r - 1) / 2 + r + 1, r + 1), na - 1);
            } else {
                r = __float2int_rz(((float)cc + 0.5f) * inv_nb);
                col = cc - r * nb;
            }
            jj = oa + r;
            kk = ob + col;
            ok = (a != b || col > r) && accept(jj, kk);
        }
        const unsigned m = __ballot_sync(FULL, ok);
        if (ok) s.tl[pos + __popc(m & ((1u << lane) - 1u))] = (unsigned)jj | ((unsigned)kk << 16);
        pos += __popc(m);
    }
    __syncwarp();
    return c;
}

/* body(jj, kk) over list entries [from, to), one entry per lane */
template <class Body>
__device__ __forceinline__ void run_list(const EfsSmem &s, int from, int to, int lane, Body body) {
    for (int t = from + lane; t < to; t += 32) {
        const unsigned pk = s.tl[t];
        body((int)(pk & 0xffffu), (int)(pk >> 16));
    }
}

/* body(jj, kk) -> the entry's force on neighbour j, over list entries
 * [from, to): each lane takes a contiguous run of K entries (K odd, so that
 * the lanes' reads of the list fall in distinct banks).  The list runs row
 * by row, so a lane's entries mostly share j: their j-side forces are summed
 * in registers and added to Fnb once per change of j.  The body must not
 * exchange values across lanes (lanes leave the loop at different times). */
template <class Body>
__device__ __forceinline__ void run_list_runs(const EfsSmem &s, int from, int to, int lane, Body body) {
    int K = (to - from + 31) >> 5;
    if (K > 0) K |= 1;
    const int t0 = from + lane * K;
    int cj = -1;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int step = 0; step < K; step++) {
        const int t = t0 + step;
        if (t >= to) break;
        const unsigned pk = s.tl[t];
        const int jj = (int)(pk & 0xffffu), kk = (int)(pk >> 16);
        if (jj != cj) {
            if (cj >= 0) {
                atomicAdd(&s.Fnb[3 * cj], -sx);
                atomicAdd(&s.Fnb[3 * cj + 1], -sy);
                atomicAdd(&s.Fnb[3 * cj + 2], -sz);
            }
            cj = jj;
            sx = sy = sz = 0.0;
        }
        const double3 g = body(jj, kk);
        sx += g.x;
        sy += g.y;
        sz += g.z;
    }
    if (cj >= 0) {
        atomicAdd(&s.Fnb[3 * cj], -sx);
        atomicAdd(&s.Fnb[3 * cj + 1], -sy);
        atomicAdd(&s.Fnb[3 * cj + 2], -sz);
    }
}

/* body(jj, kk, valid) with the whole warp converged on every round (for
 * bodies that exchange values across lanes or issue warp-wide tensor-core
 * instructions, which need all 32 lanes at one call site); lanes past the
 * end get valid = false and jj = -1 - lane, so equal jj values stay
 * adjacent */
template <class Body>
__device__ __forceinline__ void run_list_all(const EfsSmem &s, int from, int to, int lane, Body body) {
    for (int base = from; base < to; base += 32) {
        const int t = base + lane;
        const bool valid = t < to;
        const unsigned pk = valid ? s.tl[t] : 0u;
        body(valid ? (int)(pk & 0xffffu) : -1 - lane, (int)(pk >> 16), valid);
    }
}

/* Enumerate block (a,b) for this warp and process it, reusing the list
 * entries [blk[0], blk[1]) when `reuse` and filling (in rounds when the
 * region overflows) otherwise.  Records the range for later reuse and
 * returns 0 if the region overflowed (then the range is not reusable). */
/* how for_block runs a body over list entries */
enum { RUN_LANES = 0, RUN_CONVERGED = 1, RUN_RUNS = 2 };

template <int RUN, class Body>
__device__ __forceinline__ void run_entries(const EfsSmem &s, int from, int to, int lane, Body body) {
    if constexpr (RUN == RUN_CONVERGED)
        run_list_all(s, from, to, lane, body);
    else if constexpr (RUN == RUN_RUNS)
        run_list_runs(s, from, to, lane, body);
    else
        run_list(s, from, to, lane, body);
}

template <int WPA, int RUN = RUN_LANES, class Accept, class Body>
__device__ __forceinline__ int for_block(const EfsSmem &s, int a, int b, int *blk, int reuse, int &pos, int lo,
                                         int hi, int warp, int lane, Accept accept, Body body) {
    if (reuse) {
        run_entries<RUN>(s, blk[0], blk[1], lane, body);
        return 1;
    }
    int start = pos, c = warp * 32, whole = 1;
    const int C = block_candidates(s, a, b);
    for (;;) {
        const int from = pos;
        c = fill_chunks<WPA>(s, a, b, c, pos, hi, lane, accept);
        run_entries<RUN>(s, from, pos, lane, body);
        __syncwarp();
        if (c >= C) break;
        whole = 0; /* region full: restart it for the next round */
        start = pos = lo;
    }
    blk[0] = start;
    blk[1] = pos;
    return whole;
}

/* The 4-atoms-per-CTA shape holds two CTAs per SM (its shared memory per
 * atom decides that), so it may use up to 256 registers a thread: asking for
 * two blocks per SM lets it run without spills instead of the register
 * budget of three. */
template <int NE, int NZ, int NLAM, int WPA, int APB>
__global__ void __launch_bounds__(WPA * 32 * APB, APB >= 4 ? 2 : 1) k_efs(EfsArgs A) {
    constexpr int NZL = NZ * NLAM;
    constexpr int WARPS = WPA;
    constexpr int NEP = nep(NE);
    /* the reference bases (<= 8 exponents x 8 angular terms): the forward
     * grid is accumulated on the FP64 tensor cores */
    constexpr bool TC_FWD = NE <= 8 && NZL == 8;
    extern __shared__ __align__(16) char smem_raw[];
    __shared__ mb_params Ps;
    {
        const int *src = reinterpret_cast<const int *>(A.params);
        int *dst = reinterpret_cast<int *>(&Ps);
        for (int k = threadIdx.x; k < (int)(sizeof(mb_params) / sizeof(int)); k += blockDim.x) dst[k] = src[k];
        __syncthreads();
    }
    const mb_params &P = Ps;
    const int NT = WPA * 32, group = threadIdx.x / NT;
    const int tid = threadIdx.x % NT, lane = threadIdx.x & 31, warp = tid >> 5;
    const int i = blockIdx.x * APB + group;
    if (i >= A.N) return; /* whole atom groups only: no barrier spans two groups */
    const int D = P.D, ns = P.nspc, ng2 = P.ng2, ne = P.ne;
    EfsSmem s = efs_carve(smem_raw + (size_t)group * A.smem_group, A.cap, D, NE, ng2, NE * NZL, WARPS, A.tl_cap,
                          TC_FWD);
    const int tlw = A.tl_cap / WPA, tl_lo = warp * tlw, tl_hi = tl_lo + tlw;
    int tl_pos = tl_lo, tl_whole = 1;
    const int n = A.nn[i];
    const int s0 = A.spc[i];
    const double *net = A.weights + P.w_off[s0];

    /* ---- stage neighbours, stably sorted by species relative to s0 ---- */
    for (int t = tid; t < D; t += NT) s.G[t] = 0.0;
    if (warp == 0) {
        /* counts and stable ranks per relative species from warp ballots */
        const int *nj_i = A.nj + (size_t)i * A.cap;
        const unsigned below = (1u << lane) - 1u;
        int cnt[4] = {0, 0, 0, 0};
        for (int base = 0; base < n; base += 32) {
            const int t = base + lane;
            const int ds = t < n ? (A.spc[nj_i[t]] - s0 + ns) % ns : -1;
#pragma unroll
            for (int v = 0; v < 4; v++) cnt[v] += __popc(__ballot_sync(FULL, ds == v));
        }
        int off[4];
        off[0] = 0;
#pragma unroll
        for (int v = 1; v < 4; v++) off[v] = off[v - 1] + cnt[v - 1];
        if (lane < 4) {
            s.seg[lane] = cnt[lane];
            s.seg[4 + lane] = off[lane];
        }
        int run[4] = {0, 0, 0, 0};
        for (int base = 0; base < n; base += 32) {
            const int t = base + lane;
            const int j = t < n ? nj_i[t] : 0;
            const int sp = t < n ? A.spc[j] : 0;
            const int ds = t < n ? (sp - s0 + ns) % ns : -1;
            int dst = 0;
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const unsigned m = __ballot_sync(FULL, ds == v);
                if (ds == v) dst = off[v] + run[v] + __popc(m & below);
                run[v] += __popc(m);
            }
            if (t < n) {
                s.j[dst] = j;
                s.sp[dst] = sp;
                const double4 dv = A.nd[(size_t)i * A.cap + t];
                s.d[dst] = dv;
                s.ir[dst] = 1.0 / dv.w;
            }
        }
    }
    group_sync<WPA>();
    if (tid == 0 && A.counters) atomicAdd(&A.counters[0], (unsigned long long)n);

    constexpr int CELLS = ((NE * NZL + 63) / 64) * 64;
    /* list gate: the union of the forward and derivative triplet gates
     * (they coincide unless species blocks carry different cutoffs) */
    auto accept_union = [&](int jj, int kk) -> bool {
        double4 d1 = s.d[jj], d2 = s.d[kk];
        int sj = s.sp[jj], sk = s.sp[kk];
        int p01 = s0 * s0 + sj * sj, p02 = s0 * s0 + sk * sk, p12 = sj * sj + sk * sk;
        double dx = d1.x - d2.x, dy = d1.y - d2.y, dz = d1.z - d2.z;
        double r3s = dx * dx + dy * dy + dz * dz;
        bool fwd = d1.w < P.f_rc2[p01] && d1.w < P.f_rc4[p01] && d2.w < P.f_rc4[p02] && r3s < P.f_rc4sq[p12];
        bool rev = d1.w < P.d_rc4 && d2.w < P.d_rc4 && r3s < P.d_rc4sq;
        return fwd || rev;
    };
    if (A.mode != MB_MODE_VJP) {
    /* ---- forward pair terms: fc, exponential factors, G2, repulsion ---- */
    for (int t = tid; t < n; t += NT) {
        double r = s.d[t].w;
        int sj = s.sp[t], p = s0 * s0 + sj * sj;
        double fa = fcut(P.f_rc2[p], r);
        s.fa[t] = fa;
        s.fb[t] = fcut(P.f_rc4[p], r);
#pragma unroll
        for (int e = 0; e < NEP; e++)
            s.P[t * NEP + e] = e < ne ? exp(-P.f_eta4[p][e] * r * r) : 0.0;
        bool gate = r < P.f_rc2[p];
        for (int f = 0; f < ng2; f++) {
            double x = r - P.f_rs[p][f];
            s.tmp[t * ng2 + f] = gate ? fa * exp(-P.f_eta2[p][f] * (x * x)) : 0.0;
        }
    }
    group_sync<WPA>();
    /* G2 sums per relative species in neighbour order (deterministic) */
    for (int w = tid; w < ns * ng2; w += NT) {
        int v = w / ng2, f = w % ng2;
        double acc = 0.0;
        for (int t = s.seg[4 + v]; t < s.seg[4 + v] + s.seg[v]; t++) acc += s.tmp[t * ng2 + f];
        s.G[P.ind2[v] + f] = acc;
    }
    if (A.urep > 0.0 && tid == 0) {
        double eu = 0.0;
        for (int t = 0; t < n; t++) {
            double r = s.d[t].w, R = P.rm[s0] + P.rm[s.sp[t]];
            if (r < R) eu += A.urep * fcut(R, r) * R / r;
        }
        A.EU[i] = eu;
    }
    group_sync<WPA>(); /* the G2 terms in tmp are read; the triplet list reuses their space */

    /* ---- forward triplet terms, block by block of (species j, species k) ---- */
    {
        int blkid = 0;
        unsigned long long nacc = 0;
        for (int a = 0; a < ns; a++)
            for (int b = a; b < ns; b++, blkid++) {
                /* the species of j and k are fixed within the block (neighbours are
                 * sorted by species relative to s0): hoist their parameters */
                const int sja = (a + s0) % ns, skb = (b + s0) % ns;
                const int p01 = s0 * s0 + sja * sja, p02 = s0 * s0 + skb * skb, p12 = sja * sja + skb * skb;
                const double rc2_01 = P.f_rc2[p01], rc4_01 = P.f_rc4[p01], rc4_02 = P.f_rc4[p02];
                const double rc4sq_12 = P.f_rc4sq[p12], rc4_12 = P.f_rc4[p12];
                const double drc4 = P.d_rc4, drc4sq = P.d_rc4sq;
                auto accept_blk = [&](int jj, int kk) -> bool {
                    const double4 d1 = s.d[jj], d2 = s.d[kk];
                    const double dx = d1.x - d2.x, dy = d1.y - d2.y, dz = d1.z - d2.z;
                    const double r3s = dx * dx + dy * dy + dz * dz;
                    return (d1.w < rc2_01 && d1.w < rc4_01 && d2.w < rc4_02 && r3s < rc4sq_12) ||
                           (d1.w < drc4 && d2.w < drc4 && r3s < drc4sq);
                };
                const double *eta12 = P.f_eta4[p12];
                if constexpr (TC_FWD) {
                    /* Each lane takes one listed triplet and forms its 8 exponential
                     * factors ex[e] and 8 angular terms lz[zl]; the grid
                     * G[e][zl] += sum_t ex_t[e] lz_t[zl] is then an outer-product
                     * sum, done 4 triplets at a time by mma.sync m8n8k4 in FP64
                     * with the values staged through shared memory.  The
                     * accumulator fragment leaves lane l with cells 2l, 2l+1. */
                    double c0 = 0.0, c1 = 0.0;
                    double *stw = s.stage + warp * 32 * EFS_STG;
                    auto body = [&](int jj, int kk, bool valid) {
                        double ex[8], lz[NZL];
#pragma unroll
                        for (int q = 0; q < 8; q++) ex[q] = 0.0;
#pragma unroll
                        for (int q = 0; q < NZL; q++) lz[q] = 0.0;
                        if (valid) {
                            const double4 d1 = s.d[jj], d2 = s.d[kk];
                            const double dx = d1.x - d2.x, dy = d1.y - d2.y, dz = d1.z - d2.z;
                            const double r3s = dx * dx + dy * dy + dz * dz;
                            if (d1.w < rc2_01 && d1.w < rc4_01 && d2.w < rc4_02 && r3s < rc4sq_12) {
                                nacc++;
                                const double r3 = sqrt(r3s);
                                const double c = (d1.x * d2.x + d1.y * d2.y + d1.z * d2.z) * (s.ir[jj] * s.ir[kk]);
                                const double A3 = 2.0 * s.fa[jj] * s.fb[kk] * fcut(rc4_12, r3);
                                angular<NZ, NLAM>(P, c, lz, nullptr);
                                const double2 *pj = reinterpret_cast<const double2 *>(s.P + jj * NEP);
                                const double2 *pk = reinterpret_cast<const double2 *>(s.P + kk * NEP);
#pragma unroll
                                for (int h = 0; h < NEP / 2; h++) {
                                    const double2 x = pj[h], y = pk[h];
#pragma unroll
                                    for (int q = 0; q < 2; q++) {
                                        const int e = 2 * h + q;
                                        if (e < NE && e < ne)
                                            ex[e] = A3 * (q ? x.y * y.y : x.x * y.x) * exp(-eta12[e] * r3s);
                                    }
                                }
                            }
                        }
#pragma unroll
                        for (int q = 0; q < 8; q++) {
                            stw[stg_slot(lane, q)] = ex[q];
                            stw[stg_slot(lane, 8 + q)] = lz[q];
                        }
                        __syncwarp();
#pragma unroll
                        for (int st = 0; st < 8; st++) {
                            const int t = 4 * st + (lane & 3);
                            dmma884(c0, c1, stw[stg_slot(t, lane >> 2)], stw[stg_slot(t, 8 + (lane >> 2))]);
                        }
                        __syncwarp();
                    };
                    int *blk = s.blk + (blkid * WPA + warp) * 2;
                    tl_whole &= for_block<WPA, RUN_CONVERGED>(s, a, b, blk, 0, tl_pos, tl_lo, tl_hi, warp, lane, accept_blk, body);
                    group_sync<WPA>();
                    group_store64<WPA>(c0, c1, s, warp, lane);
                    {
                        /* every feature is its own descriptor entry: one per thread */
                        const int base = P.ind4[a * a + b * b];
                        for (int f = tid; f < P.ng4; f += NT)
                            s.G[base + f] += s.red[P.g4_e[f] * NZL + (P.g4_zl[f] / P.nlam) * NLAM + P.g4_zl[f] % P.nlam];
                    }
                    group_sync<WPA>();
                } else {
                double acc[CELLS];
#pragma unroll
                for (int k = 0; k < CELLS; k++) acc[k] = 0.0;
                auto body = [&](int jj, int kk) {
                    double4 d1 = s.d[jj], d2 = s.d[kk];
                    double dx = d1.x - d2.x, dy = d1.y - d2.y, dz = d1.z - d2.z;
                    double r3s = dx * dx + dy * dy + dz * dz;
                    if (!(d1.w < rc2_01 && d1.w < rc4_01 && d2.w < rc4_02 && r3s < rc4sq_12)) return;
                    nacc++;
                    double r3 = sqrt(r3s);
                    double c = (d1.x * d2.x + d1.y * d2.y + d1.z * d2.z) * (s.ir[jj] * s.ir[kk]);
                    double A3 = 2.0 * s.fa[jj] * s.fb[kk] * fcut(rc4_12, r3);
                    double lz[NZL];
#pragma unroll
                    for (int k = 0; k < NZL; k++) lz[k] = 0.0;
                    angular<NZ, NLAM>(P, c, lz, nullptr);
                    const double2 *pj = reinterpret_cast<const double2 *>(s.P + jj * NEP);
                    const double2 *pk = reinterpret_cast<const double2 *>(s.P + kk * NEP);
#pragma unroll
                    for (int h = 0; h < NEP / 2; h++) {
                        const double2 x = pj[h], y = pk[h];
#pragma unroll
                        for (int q = 0; q < 2; q++) {
                            const int e = 2 * h + q;
                            if (e >= NE || e >= ne) break;
                            const double ex = A3 * (q ? x.y * y.y : x.x * y.x) * exp(-eta12[e] * r3s);
#pragma unroll
                            for (int zl = 0; zl < NZL; zl++) acc[e * NZL + zl] += ex * lz[zl];
                        }
                    }
                };
                int *blk = s.blk + (blkid * WPA + warp) * 2;
                tl_whole &= for_block<WPA>(s, a, b, blk, 0, tl_pos, tl_lo, tl_hi, warp, lane, accept_blk, body);
                group_sync<WPA>();
#pragma unroll
                for (int ch = 0; ch < CELLS / 64; ch++) {
                    group_reduce64<WPA>(acc + 64 * ch, s, warp, lane);
                    {
                        int ds = a * a + b * b, base = P.ind4[ds];
                        for (int f = tid; f < P.ng4; f += NT) {
                            int cell = P.g4_e[f] * NZL + (P.g4_zl[f] / P.nlam) * NLAM + P.g4_zl[f] % P.nlam;
                            if (cell / 64 == ch) s.G[base + f] += s.red[cell % 64];
                        }
                    }
                    group_sync<WPA>();
                }
                }
            }
        if (A.counters) {
            for (int o = 16; o > 0; o >>= 1) nacc += __shfl_xor_sync(FULL, nacc, o);
            if (lane == 0) atomicAdd(&A.counters[1], nacc);
        }
    }

    if (A.mode == MB_MODE_DESCRIPTORS) {
        for (int t = tid; t < D; t += NT) A.G[(size_t)i * D + t] = s.G[t];
        return;
    }
    } /* end of the forward part (skipped for MB_MODE_VJP) */

    /* ---- MLP: forward (src/nmlp.c:367-431) and dE/dG ---- */
    const int h1 = P.h1, h2 = P.h2;
    const double *off = net, *W0 = off + D, *b0 = W0 + h1 * D, *W1 = b0 + h1, *b1 = W1 + h2 * h1, *W2 = b1 + h2,
                 *b2 = W2 + h2;
    double *H1 = s.h, *H2 = s.h + MB_MAXH, *Dl1 = s.h + 2 * MB_MAXH, *Dl2 = s.h + 3 * MB_MAXH;
    if (A.mode != MB_MODE_VJP) {
        for (int m = warp; m < h1; m += WARPS) {
            double acc = 0.0;
            for (int l = lane; l < D; l += 32) acc += (s.G[l] - off[l]) * W0[m * D + l];
            acc = warp_sum(acc);
            if (lane == 0) H1[m] = tanh(b0[m] + acc);
        }
        group_sync<WPA>();
        if (warp == 0) {
            double v = 0.0;
            if (lane < h2) {
                v = b1[lane];
                for (int k = 0; k < h1; k++) v += H1[k] * W1[lane * h1 + k];
                v = tanh(v);
                H2[lane] = v;
            }
            double e = lane < h2 ? v * W2[lane] : 0.0;
            e = warp_sum(e);
            if (lane == 0) A.EA[i] = b2[0] + e;
            __syncwarp();
            if (lane < h2) Dl2[lane] = W2[lane] * (1.0 - v * v);
            __syncwarp();
            if (lane < h1) {
                double g = 0.0;
                for (int m = 0; m < h2; m++) g += Dl2[m] * W1[m * h1 + lane];
                Dl1[lane] = g * (1.0 - H1[lane] * H1[lane]);
            }
        }
        group_sync<WPA>();
        if (A.mode == MB_MODE_ENERGY) return;
        /* s.G <- dE_i/dG_i */
        for (int l = tid; l < D; l += NT) {
            double g = 0.0;
            for (int k = 0; k < h1; k++) g += Dl1[k] * W0[k * D + l];
            s.G[l] = g;
        }
    } else {
        for (int l = tid; l < D; l += NT) s.G[l] = A.G[(size_t)i * D + l];
    }
    group_sync<WPA>();

    /* ---- reverse pair terms with the species-0 parameters ---- */
    double fi[3] = {0.0, 0.0, 0.0}, vr[6] = {0, 0, 0, 0, 0, 0};
    for (int t = tid; t < n; t += NT) {
        double4 d = s.d[t];
        double r = d.w, ir = 1.0 / r;
        double f4, df4, f2, df2;
        fcut_d(P.d_rc4, r, f4, df4);
        fcut_d(P.d_rc2, r, f2, df2);
        s.fa[t] = f4;
        s.fb[t] = df4;
#pragma unroll
        for (int e = 0; e < NEP; e++)
            s.P[t * NEP + e] = e < ne ? exp(-P.d_eta4[e] * r * r) : 0.0;
        int ds1 = (s.sp[t] - s0 + ns) % ns;
        const double *g = s.G + P.ind2[ds1];
        double cpair = 0.0;
        for (int f = 0; f < ng2; f++) {
            double x = r - P.d_rs[f], eta = P.d_eta2[f];
            cpair += g[f] * exp(-eta * x * x) * (-2.0 * eta * x * f2 + df2);
        }
        /* dE/dd = cpair d / r : force +on i, -on j; virial -= (dE/dd) (x) d */
        double cr = cpair * ir;
        double v0 = cr * d.x, v1 = cr * d.y, v2 = cr * d.z;
        fi[0] += v0; fi[1] += v1; fi[2] += v2;
        s.Fnb[3 * t] = -v0; s.Fnb[3 * t + 1] = -v1; s.Fnb[3 * t + 2] = -v2;
        if (A.urep > 0.0) {
            double R = P.rm[s0] + P.rm[s.sp[t]];
            if (r < R) {
                /* CELL_UREP on the ordered pair (i, j): force on i only (src/cmod.c:100-112) */
                double fu, dfu;
                fcut_d(R, r, fu, dfu);
                double tu = -2.0 * A.urep * R / (r * r) * (-fu / r + dfu);
                fi[0] -= tu * d.x; fi[1] -= tu * d.y; fi[2] -= tu * d.z;
                vr[0] += 0.5 * tu * d.x * d.x; vr[1] += 0.5 * tu * d.y * d.y; vr[2] += 0.5 * tu * d.z * d.z;
                vr[3] += 0.5 * tu * d.x * d.y; vr[4] += 0.5 * tu * d.y * d.z; vr[5] += 0.5 * tu * d.z * d.x;
            }
        }
    }
    group_sync<WPA>();

    /* ---- reverse triplet terms (list of the forward pass reused) ---- */
    {
        const int reuse = (A.mode != MB_MODE_VJP) && tl_whole;
        int blkid = 0;
        tl_pos = tl_lo;
        for (int a = 0; a < ns; a++)
            for (int b = a; b < ns; b++, blkid++) {
                const int ds = a * a + b * b, base = P.ind4[ds];
                for (int t = tid; t < NE * NZL; t += NT) s.grid[t] = 0.0;
                group_sync<WPA>();
                for (int f = tid; f < P.ng4; f += NT)
                    atomicAdd(&s.grid[P.g4_e[f] * NZL + (P.g4_zl[f] / P.nlam) * NLAM + P.g4_zl[f] % P.nlam], s.G[base + f]);
                group_sync<WPA>();
                /* returns the entry's force on neighbour j; run_list_runs sums
                 * those per lane and adds them once per change of j */
                auto body = [&](int jj, int kk) -> double3 {
                    const double4 d1 = s.d[jj], d2 = s.d[kk];
                    const double wx = d2.x - d1.x, wy = d2.y - d1.y, wz = d2.z - d1.z;
                    const double r3s = wx * wx + wy * wy + wz * wz;
                    if (!(d1.w < P.d_rc4 && d2.w < P.d_rc4 && r3s < P.d_rc4sq)) return make_double3(0.0, 0.0, 0.0);
                    double r3 = sqrt(r3s);
                    double r1 = d1.w, r2 = d2.w, ir1 = s.ir[jj], ir2 = s.ir[kk], ir3 = 1.0 / r3;
                    double c = (d1.x * d2.x + d1.y * d2.y + d1.z * d2.z) * (ir1 * ir2);
                    double f3, df3;
                    fcut_d(P.d_rc4, r3, f3, df3);
                    double f1 = s.fa[jj], df1 = s.fb[jj], f2 = s.fa[kk], df2 = s.fb[kk];
                    double lz[NZL], lzp[NZL];
#pragma unroll
                    for (int k = 0; k < NZL; k++) { lz[k] = 0.0; lzp[k] = 0.0; }
                    angular<NZ, NLAM>(P, c, lz, lzp);
                    const double2 *pj = reinterpret_cast<const double2 *>(s.P + jj * NEP);
                    const double2 *pk = reinterpret_cast<const double2 *>(s.P + kk * NEP);
                    double Q = 0.0, Qe = 0.0, Qc = 0.0;
#pragma unroll
                    for (int h = 0; h < NEP / 2; h++) {
                        const double2 x = pj[h], y = pk[h];
#pragma unroll
                        for (int q = 0; q < 2; q++) {
                            const int e = 2 * h + q;
                            if (e >= NE || e >= ne) break;
                            const double ex = (q ? x.y * y.y : x.x * y.x) * exp(-P.d_eta4[e] * r3s);
                            double u = 0.0, v = 0.0;
#pragma unroll
                            for (int zl = 0; zl < NZL; zl += 2) {
                                const double2 cg = *reinterpret_cast<const double2 *>(s.grid + e * NZL + zl);
                                u += cg.x * lz[zl] + cg.y * lz[zl + 1];
                                v += cg.x * lzp[zl] + cg.y * lzp[zl + 1];
                            }
                            Q += ex * u;
                            Qe += P.d_eta4[e] * ex * u;
                            Qc += ex * v;
                        }
                    }
                    double Af = 2.0 * f1 * f2 * f3;
                    double T1 = 2.0 * df1 * f2 * f3 * Q - 2.0 * r1 * Af * Qe;
                    double T2 = 2.0 * f1 * df2 * f3 * Q - 2.0 * r2 * Af * Qe;
                    double T3 = 2.0 * f1 * f2 * df3 * Q - 2.0 * r3 * Af * Qe;
                    double Tc = Af * Qc;
                    double a11 = T1 * ir1 - Tc * c * ir1 * ir1, a22 = T2 * ir2 - Tc * c * ir2 * ir2;
                    double a12 = Tc * ir1 * ir2, a3 = T3 * ir3;
                    const double g1x = a11 * d1.x + a12 * d2.x - a3 * wx;
                    const double g1y = a11 * d1.y + a12 * d2.y - a3 * wy;
                    const double g1z = a11 * d1.z + a12 * d2.z - a3 * wz;
                    const double g2x = a22 * d2.x + a12 * d1.x + a3 * wx;
                    const double g2y = a22 * d2.y + a12 * d1.y + a3 * wy;
                    const double g2z = a22 * d2.z + a12 * d1.z + a3 * wz;
                    fi[0] += g1x + g2x; fi[1] += g1y + g2y; fi[2] += g1z + g2z;
                    atomicAdd(&s.Fnb[3 * kk], -g2x);
                    atomicAdd(&s.Fnb[3 * kk + 1], -g2y);
                    atomicAdd(&s.Fnb[3 * kk + 2], -g2z);
                    return make_double3(g1x, g1y, g1z);
                };
                int *blk = s.blk + (blkid * WPA + warp) * 2;
                for_block<WPA, RUN_RUNS>(s, a, b, blk, reuse, tl_pos, tl_lo, tl_hi, warp, lane, accept_union, body);
                group_sync<WPA>();
            }
    }

    /* virial of atom i's energy: every neighbour force (pairs and triplets)
     * times its displacement -- the sum -(dE/dd) (x) d taken per neighbour */
    for (int t = tid; t < n; t += NT) {
        const double4 d = s.d[t];
        const double fx = s.Fnb[3 * t], fy = s.Fnb[3 * t + 1], fz = s.Fnb[3 * t + 2];
        vr[0] += fx * d.x; vr[1] += fy * d.y; vr[2] += fz * d.z;
        vr[3] += fx * d.y; vr[4] += fy * d.z; vr[5] += fz * d.x;
    }

    /* ---- write forces and the virial of atom i ---- */
    {
        double v[64];
#pragma unroll
        for (int k = 0; k < 64; k++) v[k] = 0.0;
        v[0] = fi[0]; v[1] = fi[1]; v[2] = fi[2];
#pragma unroll
        for (int k = 0; k < 6; k++) v[3 + k] = vr[k];
        group_reduce64<WPA>(v, s, warp, lane);
        if (tid == 0) {
            atomicAdd(&A.F[3 * i], s.red[0]);
            atomicAdd(&A.F[3 * i + 1], s.red[1]);
            atomicAdd(&A.F[3 * i + 2], s.red[2]);
            for (int k = 0; k < 6; k++) A.vir[(size_t)i * 6 + k] = s.red[3 + k];
        }
        for (int t = tid; t < n; t += NT) {
            int j = s.j[t];
            atomicAdd(&A.F[3 * j], s.Fnb[3 * t]);
            atomicAdd(&A.F[3 * j + 1], s.Fnb[3 * t + 1]);
            atomicAdd(&A.F[3 * j + 2], s.Fnb[3 * t + 2]);
        }
    }
}

/* ------------------------------------------------------------------ */
/* leg-table path of the descriptor pass                                */
/* ------------------------------------------------------------------ */

/* A triplet (i; j, k) of PRS_BP has three legs, i-j, i-k and j-k, and each
 * leg's factors -- exp(-eta_e r^2) for the G4 exponents and the cutoff fc(r)
 * (src/nprs.c:540-547) -- depend only on that pair.  The j-k leg is an entry
 * of j's own neighbour list, and each such entry serves every atom that has
 * both j and k as neighbours (about 29 triplets in a dense alloy).  k_legs
 * evaluates the factors once per list entry; k_efs_leg reads the j-k leg of
 * each triplet from j's row instead of evaluating it, and finds that row by
 * walking j's list and looking each entry up in a hash of i's own entries
 * keyed by (atom, image).  The walk enumerates exactly the triplets with
 * both r_ik < Rc (k is found in i's list) and r_jk < Rc (k is in j's list).
 *
 * The path applies to bases whose forward and derivative functions share one
 * cutoff and whose pair-mixed G4 exponents equal the species-0 ones (every
 * reference model; src/nprs.c:222-252 mixes identical blocks), so a leg's
 * factors serve the energy and the derivative terms alike. */

#define LEG_PER_LANE (MB_LEG_MAX_CAP / 32)
#define LEG_HASH 256 /* hash slots per atom: at least twice the neighbour capacity */


__device__ __forceinline__ unsigned hash_slot(unsigned key) { return (key * 0x9E3779B1u) >> 24; }

/* One warp per atom: sort the atom's entries stably by the neighbour's
 * species (in place: nj, nk, nd), record where each species starts
 * (nso[4i+s]; nso[4i+3] = count), write each entry's leg row with the
 * forward parameters of the pair (i, j): exp(-eta_e r^2) for e < ne (0
 * above), fc(r) and fc'(r)/r at the G4 cutoff, and put the entries' keys
 * (atom, image) with their sorted slots into the atom's hash
 * gh[i * LEG_HASH ..] (linear probing), where k_trip looks a neighbour's
 * neighbours up. */
__global__ void k_legs(int N, int cap, const int *__restrict__ nn, int *__restrict__ nj, unsigned *__restrict__ nk,
                       double4 *__restrict__ nd, const int *__restrict__ spc, const mb_params *__restrict__ Pg,
                       double *__restrict__ leg, int *__restrict__ nso, uint2 *__restrict__ gh) {
    /* the hash is built in shared memory, then copied out whole */
    __shared__ uint2 hsh[4][LEG_HASH];
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= N) return;
    const int i = warp, n = nn[i], s0 = spc[i], ne = Pg->ne;
    const size_t row = (size_t)i * cap;
    uint2 *hash = hsh[(threadIdx.x >> 5) & 3];
    for (int t = lane; t < LEG_HASH; t += 32) hash[t] = make_uint2(0xffffffffu, 0u);
    int jv[LEG_PER_LANE], spv[LEG_PER_LANE];
    unsigned kv[LEG_PER_LANE];
    double4 dv[LEG_PER_LANE];
    int cnt[MB_MAXSPC] = {0, 0, 0};
#pragma unroll
    for (int q = 0; q < LEG_PER_LANE; q++) {
        const int t = q * 32 + lane;
        spv[q] = -1;
        jv[q] = 0;
        kv[q] = 0u;
        dv[q] = make_double4(0.0, 0.0, 0.0, 1.0);
        if (t < n) {
            jv[q] = nj[row + t];
            kv[q] = nk[row + t];
            dv[q] = nd[row + t];
            spv[q] = spc[jv[q]];
        }
#pragma unroll
        for (int v = 0; v < MB_MAXSPC; v++) cnt[v] += __popc(__ballot_sync(FULL, spv[q] == v));
    }
    int off[MB_MAXSPC + 1];
    off[0] = 0;
#pragma unroll
    for (int v = 0; v < MB_MAXSPC; v++) off[v + 1] = off[v] + cnt[v];
    if (lane < 4) nso[4 * i + lane] = off[lane];
    __syncwarp();
    const unsigned below = (1u << lane) - 1u;
    int run[MB_MAXSPC] = {0, 0, 0};
#pragma unroll
    for (int q = 0; q < LEG_PER_LANE; q++) {
        int dst = 0;
#pragma unroll
        for (int v = 0; v < MB_MAXSPC; v++) {
            const unsigned m = __ballot_sync(FULL, spv[q] == v);
            if (spv[q] == v) dst = off[v] + run[v] + __popc(m & below);
            run[v] += __popc(m);
        }
        if (spv[q] >= 0) {
            nj[row + dst] = jv[q];
            nk[row + dst] = kv[q];
            nd[row + dst] = dv[q];
            {
                unsigned h = hash_slot(kv[q]);
                for (int probe = 0; probe < LEG_HASH; probe++) {
                    if (atomicCAS(&hash[h].x, 0xffffffffu, kv[q]) == 0xffffffffu) {
                        hash[h].y = (unsigned)dst;
                        break;
                    }
                    h = (h + 1u) & (LEG_HASH - 1u);
                }
            }
            const int p = s0 * s0 + spv[q] * spv[q];
            const double r = dv[q].w;
            double f, df;
            fcut_d(Pg->f_rc4[p], r, f, df);
            double e[MB_LEG_STRIDE];
#pragma unroll
            for (int k = 0; k < 8; k++) e[k] = k < ne ? exp(-Pg->f_eta4[p][k] * r * r) : 0.0;
            e[8] = f;
            e[9] = df / r;
            /* with at most 7 exponents slot 7 is free: fc again, so that the
             * forward pass reads 4 of a row's 5 16-byte pieces */
            if (ne <= 7) e[7] = f;
            double2 *o = reinterpret_cast<double2 *>(leg + (row + dst) * MB_LEG_STRIDE);
#pragma unroll
            for (int k = 0; k < MB_LEG_STRIDE / 2; k++) o[k] = make_double2(e[2 * k], e[2 * k + 1]);
        }
    }
    __syncwarp();
    uint2 *out = gh + (size_t)i * LEG_HASH;
    for (int t = lane; t < LEG_HASH; t += 32) out[t] = hash[t];
}

struct LegArgs {
    int N, cap, mode;
    double urep;
    const int *nn, *nj, *nso;
    const double4 *nd;
    const double *leg;
    const uint2 *trip; /* triplet lists (k_trip) */
    const int *tboff;
    int tcap;
    const int *spc;
    const mb_params *params;
    const double *weights;
    double *EA, *EU, *G, *F, *vir;
    unsigned long long *counters;
    size_t smem_group;
    mb_params P; /* by value: read from the kernel-parameter space through the constant cache */
};

/* Row of one list entry in k_efs_leg's shared memory: x, y, z, 1/r as two
 * 16-byte loads, then r and a pad.  At 48 bytes a row, the 16-byte loads
 * of 8 consecutive entries (a quarter-warp) fall in distinct banks; rows of
 * 32 bytes (a double4) conflicted 2-way. */
#define LEG_DROW 6
__device__ __forceinline__ double4 leg_vec(const double *d, int u) {
    const double2 *p = reinterpret_cast<const double2 *>(d + LEG_DROW * u);
    const double2 a = p[0], b = p[1];
    return make_double4(a.x, a.y, b.x, b.y);
}

/* shared-memory carve-up of one atom group of k_efs_leg */
struct LegSmem {
    double *stage;                          /* tensor-core staging (forward) | */
    double *Fnb, *grid, *red, *h;           /* reductions, MLP, reverse pass   */
    double *d;                              /* per entry x, y, z, 1/r, r, 0    */
    double *L, *G;
    double *tmp;                            /* G2 terms (in the stage region) */
    int *j, *sp, *seg;
};

/* The G2 terms (tmp) are read before the forward triplets start, so they
 * share the region of the staging rows and the later reductions. */
__host__ __device__ inline size_t leg_union_bytes(int cap, int ng2, int warps) {
    const size_t u = efs_union_bytes(cap, 64, warps, 1), t = align16(sizeof(double) * cap * (ng2 > 1 ? ng2 : 1));
    return u > t ? u : t;
}

__host__ __device__ inline size_t leg_smem_bytes(int cap, int D, int ng2, int warps) {
    size_t b = leg_union_bytes(cap, ng2, warps);
    b += sizeof(double) * cap * LEG_DROW;                      /* d */
    b += sizeof(double) * cap * MB_LEG_STRIDE;                 /* L */
    b += align16(sizeof(double) * D);                          /* G */
    b += align16(sizeof(int) * cap) * 2;                       /* j, sp */
    b += sizeof(int) * 8;                                      /* seg */
    return align16(b);
}

__device__ inline LegSmem leg_carve(char *base, int cap, int D, int ng2, int warps) {
    LegSmem s;
    char *p = base;
    s.stage = (double *)p;
    s.Fnb = (double *)p;
    s.grid = s.Fnb + cap * 3;
    s.red = s.grid + 64;
    s.h = s.red + warps * 64;
    s.tmp = (double *)p;
    p += leg_union_bytes(cap, ng2, warps);
    s.d = (double *)p; p += sizeof(double) * cap * LEG_DROW;
    s.L = (double *)p; p += sizeof(double) * cap * MB_LEG_STRIDE;
    s.G = (double *)p; p += align16(sizeof(double) * D);
    s.j = (int *)p; p += align16(sizeof(int) * cap);
    s.sp = (int *)p; p += align16(sizeof(int) * cap);
    s.seg = (int *)p;
    return s;
}


/* Triplet lists of the leg path: one warp per atom i, TRIP_WARPS atoms per
 * CTA.  PRS_BP takes the triplet (j, k) of i when NDX[i][j] and NDX[i][k]
 * are below the G4 cutoff and so is ndx[i][j][k] = |DX_j - DX_k|, both
 * displacements from i's list (src/nprs.c:528-537, src/cell.c:175-181).
 * The warp stages i's entries in relative-species order (position u, the
 * order k_efs_leg stages them in: relative species v holds absolute
 * species (s0 + v) % ns) and walks, per species block (alpha <= beta), the
 * pairs (a, b), b > a, 32 per round, with that test: the squared distance
 * summed without contraction as the reference forms it, compared with the
 * threshold for which sqrt(s) < Rc holds exactly.  An accepted pair's j-k
 * leg row is the entry of k (its atom at the image shift(b) - shift(a)) in
 * j's own list, found in j's hash (k_legs); a pair whose k is not in j's
 * list lies within rounding of the cutoff, where fc vanishes, and is left
 * out.  Entries {a | b << 8, j cap + c} are written in pair order (a, then
 * b), so every list is deterministic and at most cap (cap - 1) / 2 long;
 * tboff[8 i + blk] holds each block's start and tboff[8 i + nblk] the end.
 * counters[1] (if set) receives the number of triplets. */
/* 4 atoms per CTA: the CTAs all fit in one wave either way, and with
 * smaller CTAs the SMs' shares of the 4000-atom alloy differ by 4 warps
 * instead of 8 (about 7 us faster a pass than 8 atoms per CTA; 2 per CTA
 * was no faster than 4) */
#define TRIP_WARPS 4

/* The 15-bit image field of an entry key (three 5-bit two's-complement
 * shifts) as three biased (x + 16) 7-bit fields, so that shifts add and
 * subtract as integers. */
__device__ __forceinline__ unsigned spread_img(unsigned key) {
    const unsigned f = (key & 0x7fffu) ^ 0x4210u; /* x + 16 per field */
    return (f & 31u) | ((f & (31u << 5)) << 2) | ((f & (31u << 10)) << 4);
}
#define IMG_48 (48u | (48u << 7) | (48u << 14))
#define IMG_BIT5 ((1u << 5) | (1u << 12) | (1u << 19))
#define IMG_BIT6 ((1u << 6) | (1u << 13) | (1u << 20))

__global__ void __launch_bounds__(32 * TRIP_WARPS) k_trip(int N, int cap, int tcap, int ns, const int *__restrict__ nn,
                                                          const int *__restrict__ nj, const unsigned *__restrict__ nk,
                                                          const double4 *__restrict__ nd, const int *__restrict__ nso,
                                                          const int *__restrict__ spc, const mb_params *__restrict__ Pg,
                                                          const uint2 *__restrict__ gh, uint2 *__restrict__ trip,
                                                          int *__restrict__ tboff, unsigned long long *counters) {
    __shared__ double4 sd[TRIP_WARPS][MB_LEG_MAX_CAP];
    __shared__ unsigned skey[TRIP_WARPS][MB_LEG_MAX_CAP];
    __shared__ int sj[TRIP_WARPS][MB_LEG_MAX_CAP];
    __shared__ int sseg[TRIP_WARPS][8];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * TRIP_WARPS + w;
    if (i >= N) return; /* whole warps; nothing below synchronises the CTA */
    double4 *d = sd[w];
    unsigned *key = skey[w];
    int *js = sj[w], *seg = sseg[w];
    const int n = nn[i], s0 = spc[i];
    const size_t row = (size_t)i * cap;
    if (lane < 4) {
        const int v = lane, sa = (s0 + v) % ns;
        int c = 0, o = 0;
        if (v < ns) c = nso[4 * i + sa + 1] - nso[4 * i + sa];
        for (int u = 0; u < v; u++) {
            const int su = (s0 + u) % ns;
            o += nso[4 * i + su + 1] - nso[4 * i + su];
        }
        seg[v] = c;
        seg[4 + v] = v < ns ? o : n;
    }
    __syncwarp();
    for (int u = lane; u < n; u += 32) {
        int v = 0;
        while (v + 1 < ns && u >= seg[4 + v + 1]) v++;
        const int sa = (s0 + v) % ns;
        const int t = nso[4 * i + sa] + (u - seg[4 + v]);
        d[u] = nd[row + t];
        key[u] = nk[row + t];
        js[u] = nj[row + t];
    }
    __syncwarp();
    uint2 *out = trip + (size_t)i * tcap;
    int pos = 0, blkid = 0;
    for (int al = 0; al < ns; al++)
        for (int be = al; be < ns; be++, blkid++) {
            if (lane == 0) tboff[8 * i + blkid] = pos;
            const int sj_ = (s0 + al) % ns, sk_ = (s0 + be) % ns;
            const int p01 = s0 * s0 + sj_ * sj_, p02 = s0 * s0 + sk_ * sk_, p12 = sj_ * sj_ + sk_ * sk_;
            const double R01 = __ldg(&Pg->f_rc4[p01]), R02 = __ldg(&Pg->f_rc4[p02]);
            const double thr = __ldg(&Pg->f_rc4thr[p12]);
            const int na = seg[al], nb = seg[be], oa = seg[4 + al], ob = seg[4 + be];
            const bool tri = al == be;
            const int C = tri ? na * (na - 1) / 2 : na * nb;
            /* the lane's candidates are c = lane, lane + 32, ...: candidate c
             * is row r, position p of the block (row r of the strict upper
             * triangle holds na - 1 - r pairs starting at column r + 1; a
             * rectangular block's rows hold nb), and the cursor (r, p)
             * moves on by 32 per candidate; it never passes the last row */
            const int rmax = tri ? na - 2 : na - 1;
            int r = 0, p = lane;
            if (C > 0)
                while (p >= (tri ? na - 1 - r : nb) && r < rmax) {
                    p -= tri ? na - 1 - r : nb;
                    r++;
                }
            /* two candidate pairs per lane and iteration (c and c + 32): both
             * first hash probes are in flight together; entries are still
             * written in candidate order */
            for (int base = 0; base < C; base += 64) {
                unsigned kk[2], h[2], ax[2], jx[2];
                const uint2 *hj[2];
                bool live[2];
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    const int c = base + 32 * q + lane;
                    live[q] = false;
                    kk[q] = 0u;
                    h[q] = 0u;
                    ax[q] = 0u;
                    jx[q] = 0u;
                    hj[q] = gh;
                    if (c < C) {
                        const int col = tri ? r + 1 + p : p;
                        const int a = oa + r, b = ob + col;
                        const double4 da = d[a], db = d[b];
                        const double dx = xsub(da.x, db.x), dy = xsub(da.y, db.y), dz = xsub(da.z, db.z);
                        const double s2 = xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
                        if (da.w < R01 && db.w < R02 && s2 < thr) {
                            const unsigned ka = key[a], kb = key[b];
                            const unsigned t = IMG_48 + spread_img(kb) - spread_img(ka);
                            if ((t & IMG_BIT6) == 0u && (t & IMG_BIT5) == IMG_BIT5) {
                                const unsigned f = (t & 31u) | ((t >> 2) & (31u << 5)) | ((t >> 4) & (31u << 10));
                                kk[q] = (kb & ~0x7fffu) | (f ^ 0x4210u); /* k at its image relative to j */
                                const int j = js[a];
                                jx[q] = (unsigned)j;
                                hj[q] = gh + (size_t)j * LEG_HASH;
                                h[q] = hash_slot(kk[q]);
                                ax[q] = (unsigned)a | ((unsigned)b << 8);
                                live[q] = true;
                            }
                        }
                    }
                    p += 32;
                    while (p >= (tri ? na - 1 - r : nb) && r < rmax) {
                        p -= tri ? na - 1 - r : nb;
                        r++;
                    }
                }
                uint2 e[2];
#pragma unroll
                for (int q = 0; q < 2; q++) e[q] = live[q] ? __ldg(hj[q] + h[q]) : make_uint2(0xffffffffu, 0u);
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    bool ok = false;
                    uint2 ent = make_uint2(0u, 0u);
                    if (live[q]) {
                        /* the first probe is in e[q]; at most LEG_HASH probes in all */
                        uint2 x = e[q];
                        unsigned hq = h[q];
                        for (int probe = 0; probe < LEG_HASH; probe++) {
                            if (x.x == kk[q]) {
                                ok = true;
                                ent = make_uint2(ax[q], jx[q] * (unsigned)cap + x.y);
                                break;
                            }
                            if (x.x == 0xffffffffu) break;
                            hq = (hq + 1u) & (LEG_HASH - 1u);
                            x = __ldg(hj[q] + hq);
                        }
                    }
                    const unsigned m = __ballot_sync(FULL, ok);
                    if (ok) out[pos + __popc(m & ((1u << lane) - 1u))] = ent;
                    pos += __popc(m);
                }
            }
        }
    if (lane == 0) {
        tboff[8 * i + blkid] = pos;
        if (counters) atomicAdd(&counters[1], (unsigned long long)pos);
    }
}

/* body(ent) -> the entry's force on neighbour a, over list entries
 * [from, to): each lane takes a contiguous run of K entries (K odd);
 * consecutive entries mostly share a, so the a-side forces are summed in
 * registers and added to Fnb once per change of a. */
template <class Body>
__device__ __forceinline__ void leg_run_runs(const LegSmem &s, const uint2 *__restrict__ list, int from, int to,
                                             int lane, Body body) {
    int K = (to - from + 31) >> 5;
    if (K > 0) K |= 1;
    const int t0 = from + lane * K, t1 = min(to, t0 + K);
    int ca = -1;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    uint2 nxt = t0 < t1 ? __ldg(list + t0) : make_uint2(0u, 0u);
    for (int t = t0; t < t1; t++) {
        const uint2 ent = nxt;
        if (t + 1 < t1) nxt = __ldg(list + t + 1); /* the next entry is in flight while this one is computed */
        const int a = (int)(ent.x & 0xffu);
        if (a != ca) {
            if (ca >= 0) {
                atomicAdd(&s.Fnb[3 * ca], -sx);
                atomicAdd(&s.Fnb[3 * ca + 1], -sy);
                atomicAdd(&s.Fnb[3 * ca + 2], -sz);
            }
            ca = a;
            sx = sy = sz = 0.0;
        }
        const double3 g = body(ent);
        sx += g.x;
        sy += g.y;
        sz += g.z;
    }
    if (ca >= 0) {
        atomicAdd(&s.Fnb[3 * ca], -sx);
        atomicAdd(&s.Fnb[3 * ca + 1], -sy);
        atomicAdd(&s.Fnb[3 * ca + 2], -sz);
    }
}

/* body(ent) -> the entry's force on neighbour a, over list entries
 * [from, to), 32 consecutive entries per round (the forward pass's
 * layout): a block's entries are ordered by a, so within a round the lanes
 * of one a are contiguous and their b slots all differ (few conflicting
 * b-side atomics); the a-side forces are summed per run of equal a by a
 * segmented warp sum and added by the run's first lane. */
template <class Body>
__device__ __forceinline__ void leg_run_conv(const LegSmem &s, const uint2 *__restrict__ list, int from, int to,
                                             int lane, Body body) {
    uint2 cur = from + lane < to ? __ldg(list + from + lane) : make_uint2(0u, 0u);
    for (int base = from; base < to; base += 32) {
        const int t = base + lane, tn = t + 32;
        const uint2 nxt = tn < to ? __ldg(list + tn) : make_uint2(0u, 0u);
        const bool valid = t < to;
        const int a = valid ? (int)(cur.x & 0xffu) : 256 + lane; /* idle lanes: segments of their own */
        double3 g = valid ? body(cur) : make_double3(0.0, 0.0, 0.0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double x = __shfl_down_sync(FULL, g.x, o), y = __shfl_down_sync(FULL, g.y, o),
                         z = __shfl_down_sync(FULL, g.z, o);
            const int an = __shfl_down_sync(FULL, a, o);
            if (lane + o < 32 && an == a) {
                g.x += x;
                g.y += y;
                g.z += z;
            }
        }
        const int ap = __shfl_up_sync(FULL, a, 1);
        if (valid && (lane == 0 || ap != a)) {
            atomicAdd(&s.Fnb[3 * a], -g.x);
            atomicAdd(&s.Fnb[3 * a + 1], -g.y);
            atomicAdd(&s.Fnb[3 * a + 2], -g.z);
        }
        cur = nxt;
    }
}

/* The fused descriptor / MLP / force kernel on leg tables: the stages of
 * k_efs over the triplet lists of k_trip, with every triplet's leg factors
 * read from the rows k_legs wrote (i-j and i-k from i's own rows, staged;
 * j-k from j's row in global memory, L2-resident).  Reference bases: at
 * most 8 G4 exponents, zeta in {1, 2, 4, 16} or other integers, 2 lambdas. */
/* Register budget per shape: the multi-warp shapes are compiled for 16
 * resident warps per SM (at most 128 registers a thread; a few bytes of
 * spills, measured 3-9% faster than 12 warps), the one-warp shapes for 12
 * (their shared memory allows no more at the alloy's neighbour counts).
 * RV selects the reverse pass's layout: 0 per-lane runs of entries (a-side
 * forces in registers), 1 consecutive entries per round (b-side atomics
 * without conflicts within a row). */
template <int NE, int WPA, int APB, int RV>
__global__ void __launch_bounds__(WPA * 32 * APB, (WPA >= 2 ? 512 : 384) / (WPA * 32 * APB))
    k_efs_leg(const __grid_constant__ LegArgs A) {
    constexpr int NZ = 4, NLAM = 2, NZL = 8;
    static_assert(NE == 7 || NE == 8, "leg rows hold 8 exponents");
    extern __shared__ __align__(16) char smem_raw[];
    const mb_params &P = A.P;
    /* G4 feature -> cell of the (eta, zeta-lambda) grid: the one table read
     * at a different index by every thread, so it is kept in shared memory */
    __shared__ unsigned char g4cell[MB_MAXG4];
    for (int f = threadIdx.x; f < P.ng4; f += blockDim.x)
        g4cell[f] = (unsigned char)(P.g4_e[f] * NZL + (P.g4_zl[f] / P.nlam) * NLAM + P.g4_zl[f] % P.nlam);
    __syncthreads();
    const int NT = WPA * 32, group = threadIdx.x / NT;
    const int tid = threadIdx.x % NT, lane = threadIdx.x & 31, warp = tid >> 5;
    const int i = blockIdx.x * APB + group;
    if (i >= A.N) return; /* whole atom groups only: no barrier spans two groups */
    const int D = P.D, ns = P.nspc, ng2 = P.ng2, ne = P.ne, cap = A.cap;
    LegSmem s = leg_carve(smem_raw + (size_t)group * A.smem_group, cap, D, ng2, WPA);
    const uint2 *tl = A.trip + (size_t)i * A.tcap;
    const int *tb = A.tboff + 8 * (size_t)i;
    const int n = A.nn[i];
    const int s0 = A.spc[i];
    const double *net = A.weights + P.w_off[s0];
    const size_t row = (size_t)i * cap;

    /* ---- stage i's entries in relative-species order (k_legs sorted them by
     * absolute species: relative species v is absolute (s0 + v) % ns) ---- */
    if (tid < 4) {
        const int v = tid, sa = (s0 + v) % ns;
        int c = 0, o = 0;
        if (v < ns) c = A.nso[4 * i + sa + 1] - A.nso[4 * i + sa];
        for (int w = 0; w < v; w++) {
            const int sw = (s0 + w) % ns;
            o += A.nso[4 * i + sw + 1] - A.nso[4 * i + sw];
        }
        s.seg[v] = c;
        s.seg[4 + v] = v < ns ? o : n;
    }
    for (int t = tid; t < D; t += NT) s.G[t] = 0.0;
    group_sync<WPA>();
    for (int u = tid; u < n; u += NT) {
        int v = 0;
        while (v + 1 < ns && u >= s.seg[4 + v + 1]) v++;
        const int sa = (s0 + v) % ns;
        const int t = A.nso[4 * i + sa] + (u - s.seg[4 + v]);
        const int j = A.nj[row + t];
        const double4 dv = A.nd[row + t];
        s.j[u] = j;
        s.sp[u] = sa;
        double2 *dr = reinterpret_cast<double2 *>(s.d + LEG_DROW * u);
        dr[0] = make_double2(dv.x, dv.y);
        dr[1] = make_double2(dv.z, 1.0 / dv.w);
        dr[2] = make_double2(dv.w, 0.0);
        const double2 *src = reinterpret_cast<const double2 *>(A.leg + (row + t) * MB_LEG_STRIDE);
        double2 *dst = reinterpret_cast<double2 *>(s.L + (size_t)u * MB_LEG_STRIDE);
#pragma unroll
        for (int k = 0; k < MB_LEG_STRIDE / 2; k++) dst[k] = __ldg(src + k);
    }
    group_sync<WPA>();
    if (tid == 0 && A.counters) atomicAdd(&A.counters[0], (unsigned long long)n);

    if (A.mode != MB_MODE_VJP) {
        /* ---- forward pair terms: G2 (src/nprs.c:518-526) and repulsion ---- */
        for (int t = tid; t < n; t += NT) {
            const double r = s.d[LEG_DROW * t + 4];
            const int p = s0 * s0 + s.sp[t] * s.sp[t];
            const double fa = s.L[t * MB_LEG_STRIDE + 8]; /* one cutoff for all functions */
            for (int f = 0; f < ng2; f++) {
                const double x = r - P.f_rs[p][f];
                s.tmp[t * ng2 + f] = fa * exp(-P.f_eta2[p][f] * (x * x));
            }
        }
        group_sync<WPA>();
        for (int w = tid; w < ns * ng2; w += NT) {
            const int v = w / ng2, f = w % ng2;
            double acc = 0.0;
            for (int t = s.seg[4 + v]; t < s.seg[4 + v] + s.seg[v]; t++) acc += s.tmp[t * ng2 + f];
            s.G[P.ind2[v] + f] = acc;
        }
        if (A.urep > 0.0 && tid == 0) {
            double eu = 0.0;
            for (int t = 0; t < n; t++) {
                const double r = s.d[LEG_DROW * t + 4], R = P.rm[s0] + P.rm[s.sp[t]];
                if (r < R) eu += A.urep * fcut(R, r) * R / r;
            }
            A.EU[i] = eu;
        }
        group_sync<WPA>(); /* the G2 terms in tmp are read; the triplet list reuses their space */

        /* ---- forward triplet terms, block by block, on the FP64 tensor cores ---- */
        int blkid = 0;
        for (int al = 0; al < ns; al++)
            for (int be = al; be < ns; be++, blkid++) {
                double c0 = 0.0, c1 = 0.0;
                double *stw = s.stage + warp * 32 * EFS_STG;
                auto body = [&](uint2 ent, bool valid) {
                    double ex[8], lz[NZL];
#pragma unroll
                    for (int q = 0; q < 8; q++) ex[q] = 0.0;
#pragma unroll
                    for (int q = 0; q < NZL; q++) lz[q] = 0.0;
                    if (valid) {
                        const int a = (int)(ent.x & 0xffu), b = (int)((ent.x >> 8) & 0xffu);
                        const double4 d1 = leg_vec(s.d, a), d2 = leg_vec(s.d, b);
                        const double c = (d1.x * d2.x + d1.y * d2.y + d1.z * d2.z) * (d1.w * d2.w);
                        const double2 *la = reinterpret_cast<const double2 *>(s.L + a * MB_LEG_STRIDE);
                        const double2 *lb = reinterpret_cast<const double2 *>(s.L + b * MB_LEG_STRIDE);
                        const double2 *lg = reinterpret_cast<const double2 *>(A.leg + (size_t)ent.y * MB_LEG_STRIDE);
                        /* fc of the three legs: slot 7 when it is free (NE = 7), else slot 8 */
                        const double A3 = NE == 7 ? 2.0 * la[3].y * lb[3].y * __ldg(lg + 3).y
                                                  : 2.0 * la[4].x * lb[4].x * __ldg(lg + 4).x;
                        angular<NZ, NLAM, false>(P, c, lz, nullptr);
#pragma unroll
                        for (int hh = 0; hh < (NE + 1) / 2; hh++) {
                            const double2 x = la[hh], y = lb[hh], z = __ldg(lg + hh);
                            ex[2 * hh] = A3 * (x.x * y.x) * z.x;
                            if (2 * hh + 1 < NE) ex[2 * hh + 1] = A3 * (x.y * y.y) * z.y;
                        }
                    }
#pragma unroll
                    for (int q = 0; q < 8; q++) {
                        stw[stg_slot(lane, q)] = ex[q];
                        stw[stg_slot(lane, 8 + q)] = lz[q];
                    }
                    __syncwarp();
#pragma unroll
                    for (int st = 0; st < 8; st++) {
                        const int t = 4 * st + (lane & 3);
                        dmma884(c0, c1, stw[stg_slot(t, lane >> 2)], stw[stg_slot(t, 8 + (lane >> 2))]);
                    }
                    __syncwarp();
                };
                /* the block's list entries, 32 per round, the atom's warps taking every WPA-th round */
                {
                    const int to = tb[blkid + 1];
                    int base = tb[blkid] + warp * 32;
                    uint2 cur = base + lane < to ? __ldg(tl + base + lane) : make_uint2(0u, 0u);
                    for (; base < to; base += 32 * WPA) {
                        /* the next round's entry is in flight while this round is computed */
                        const int tn = base + 32 * WPA + lane;
                        const uint2 nxt = tn < to ? __ldg(tl + tn) : make_uint2(0u, 0u);
                        body(cur, base + lane < to);
                        cur = nxt;
                    }
                }
                group_sync<WPA>();
                group_store64<WPA>(c0, c1, s, warp, lane);
                {
                    const int base = P.ind4[al * al + be * be];
                    /* the cells carry the zeta normalisation left out of the angular terms */
                    for (int f = tid; f < P.ng4; f += NT)
                        s.G[base + f] += s.red[g4cell[f]] * P.powz[(g4cell[f] & 7) >> 1];
                }
                group_sync<WPA>();
            }
        if (A.mode == MB_MODE_DESCRIPTORS) {
            for (int t = tid; t < D; t += NT) A.G[(size_t)i * D + t] = s.G[t];
            return;
        }
    }

    /* ---- MLP: forward (src/nmlp.c:367-431) and dE/dG ---- */
    const int h1 = P.h1, h2 = P.h2;
    const double *off = net, *W0 = off + D, *b0 = W0 + h1 * D, *W1 = b0 + h1, *b1 = W1 + h2 * h1, *W2 = b1 + h2,
                 *b2 = W2 + h2;
    double *H1 = s.h, *H2 = s.h + MB_MAXH, *Dl1 = s.h + 2 * MB_MAXH, *Dl2 = s.h + 3 * MB_MAXH;
    if (A.mode != MB_MODE_VJP) {
        for (int m = warp; m < h1; m += WPA) {
            double acc = 0.0;
            for (int l = lane; l < D; l += 32) acc += (s.G[l] - off[l]) * W0[m * D + l];
            acc = warp_sum(acc);
            if (lane == 0) H1[m] = tanh(b0[m] + acc);
        }
        group_sync<WPA>();
        if (warp == 0) {
            double v = 0.0;
            if (lane < h2) {
                v = b1[lane];
                for (int k = 0; k < h1; k++) v += H1[k] * W1[lane * h1 + k];
                v = tanh(v);
                H2[lane] = v;
            }
            double e = lane < h2 ? v * W2[lane] : 0.0;
            e = warp_sum(e);
            if (lane == 0) A.EA[i] = b2[0] + e;
            __syncwarp();
            if (lane < h2) Dl2[lane] = W2[lane] * (1.0 - v * v);
            __syncwarp();
            if (lane < h1) {
                double g = 0.0;
                for (int m = 0; m < h2; m++) g += Dl2[m] * W1[m * h1 + lane];
                Dl1[lane] = g * (1.0 - H1[lane] * H1[lane]);
            }
        }
        group_sync<WPA>();
        if (A.mode == MB_MODE_ENERGY) return;
        for (int l = tid; l < D; l += NT) {
            double g = 0.0;
            for (int k = 0; k < h1; k++) g += Dl1[k] * W0[k * D + l];
            s.G[l] = g;
        }
    } else {
        for (int l = tid; l < D; l += NT) s.G[l] = A.G[(size_t)i * D + l];
    }
    group_sync<WPA>();

    /* ---- reverse pair terms with the species-0 parameters ---- */
    double fi[3] = {0.0, 0.0, 0.0}, vr[6] = {0, 0, 0, 0, 0, 0};
    for (int t = tid; t < n; t += NT) {
        const double4 d = leg_vec(s.d, t);
        const double r = s.d[LEG_DROW * t + 4], ir = d.w;
        double f2, df2;
        fcut_d(P.d_rc2, r, f2, df2);
        const int ds1 = (s.sp[t] - s0 + ns) % ns;
        const double *g = s.G + P.ind2[ds1];
        double cpair = 0.0;
        for (int f = 0; f < ng2; f++) {
            const double x = r - P.d_rs[f], eta = P.d_eta2[f];
            cpair += g[f] * exp(-eta * x * x) * (-2.0 * eta * x * f2 + df2);
        }
        const double cr = cpair * ir;
        const double v0 = cr * d.x, v1 = cr * d.y, v2 = cr * d.z;
        fi[0] += v0; fi[1] += v1; fi[2] += v2;
        s.Fnb[3 * t] = -v0; s.Fnb[3 * t + 1] = -v1; s.Fnb[3 * t + 2] = -v2;
        if (A.urep > 0.0) {
            const double R = P.rm[s0] + P.rm[s.sp[t]];
            if (r < R) {
                /* CELL_UREP on the ordered pair (i, j): force on i only (src/cmod.c:100-112) */
                double fu, dfu;
                fcut_d(R, r, fu, dfu);
                const double tu = -2.0 * A.urep * R / (r * r) * (-fu / r + dfu);
                fi[0] -= tu * d.x; fi[1] -= tu * d.y; fi[2] -= tu * d.z;
                vr[0] += 0.5 * tu * d.x * d.x; vr[1] += 0.5 * tu * d.y * d.y; vr[2] += 0.5 * tu * d.z * d.z;
                vr[3] += 0.5 * tu * d.x * d.y; vr[4] += 0.5 * tu * d.y * d.z; vr[5] += 0.5 * tu * d.z * d.x;
            }
        }
    }
    group_sync<WPA>();

    /* ---- reverse triplet terms over the same lists ---- */
    {
        int blkid = 0;
        double eta[NE];
#pragma unroll
        for (int e = 0; e < NE; e++) eta[e] = e < ne ? P.d_eta4[e] : 0.0;
        for (int al = 0; al < ns; al++)
            for (int be = al; be < ns; be++, blkid++) {
                const int base = P.ind4[al * al + be * be];
                for (int t = tid; t < 64; t += NT) s.grid[t] = 0.0;
                group_sync<WPA>();
                for (int f = tid; f < P.ng4; f += NT)
                    atomicAdd(&s.grid[g4cell[f]], s.G[base + f] * P.powz[(g4cell[f] & 7) >> 1]);
                group_sync<WPA>();
                auto body = [&](uint2 ent) -> double3 {
                    const int a = (int)(ent.x & 0xffu), b = (int)((ent.x >> 8) & 0xffu);
                    const double4 d1 = leg_vec(s.d, a), d2 = leg_vec(s.d, b);
                    const double wx = d2.x - d1.x, wy = d2.y - d1.y, wz = d2.z - d1.z;
                    const double ir1 = d1.w, ir2 = d2.w;
                    const double c = (d1.x * d2.x + d1.y * d2.y + d1.z * d2.z) * (ir1 * ir2);
                    const double2 *la = reinterpret_cast<const double2 *>(s.L + a * MB_LEG_STRIDE);
                    const double2 *lb = reinterpret_cast<const double2 *>(s.L + b * MB_LEG_STRIDE);
                    const double2 *lg = reinterpret_cast<const double2 *>(A.leg + (size_t)ent.y * MB_LEG_STRIDE);
                    const double2 fa = la[4], fb = lb[4], fg = __ldg(lg + 4);
                    double lz[NZL], lzp[NZL];
#pragma unroll
                    for (int k = 0; k < NZL; k++) { lz[k] = 0.0; lzp[k] = 0.0; }
                    angular<NZ, NLAM, false>(P, c, lz, lzp);
                    double Q = 0.0, Qe = 0.0, Qc = 0.0;
#pragma unroll
                    for (int hh = 0; hh < (NE + 1) / 2; hh++) {
                        const double2 x = la[hh], y = lb[hh], z = __ldg(lg + hh);
#pragma unroll
                        for (int q = 0; q < 2; q++) {
                            const int e = 2 * hh + q;
                            if (e >= NE) break;
                            const double E = q ? (x.y * y.y) * z.y : (x.x * y.x) * z.x;
                            double u = 0.0, v = 0.0;
#pragma unroll
                            for (int zl = 0; zl < NZL; zl += 2) {
                                const double2 cg = *reinterpret_cast<const double2 *>(s.grid + e * NZL + zl);
                                u += cg.x * lz[zl] + cg.y * lz[zl + 1];
                                v += cg.x * lzp[zl] + cg.y * lzp[zl + 1];
                            }
                            Q += E * u;
                            Qe += eta[e] * E * u;
                            Qc += E * v;
                        }
                    }
                    /* legs: f = fc(r), h = fc'(r)/r (i-j: a, i-k: b, j-k: g) */
                    const double Af = 2.0 * fa.x * fb.x * fg.x;
                    const double T1 = 2.0 * fa.y * fb.x * fg.x * Q - 2.0 * Af * Qe; /* dT/dr1 / r1 */
                    const double T2 = 2.0 * fa.x * fb.y * fg.x * Q - 2.0 * Af * Qe;
                    const double T3 = 2.0 * fa.x * fb.x * fg.y * Q - 2.0 * Af * Qe;
                    const double Tc = Af * Qc;
                    const double a11 = T1 - Tc * c * ir1 * ir1, a22 = T2 - Tc * c * ir2 * ir2;
                    const double a12 = Tc * ir1 * ir2, a3 = T3;
                    const double g1x = a11 * d1.x + a12 * d2.x - a3 * wx;
                    const double g1y = a11 * d1.y + a12 * d2.y - a3 * wy;
                    const double g1z = a11 * d1.z + a12 * d2.z - a3 * wz;
                    const double g2x = a22 * d2.x + a12 * d1.x + a3 * wx;
                    const double g2y = a22 * d2.y + a12 * d1.y + a3 * wy;
                    const double g2z = a22 * d2.z + a12 * d1.z + a3 * wz;
                    fi[0] += g1x + g2x; fi[1] += g1y + g2y; fi[2] += g1z + g2z;
                    atomicAdd(&s.Fnb[3 * b], -g2x);
                    atomicAdd(&s.Fnb[3 * b + 1], -g2y);
                    atomicAdd(&s.Fnb[3 * b + 2], -g2z);
                    return make_double3(g1x, g1y, g1z);
                };
                {
                    /* the block's entries in WPA contiguous parts, one per warp */
                    const int from = tb[blkid], to = tb[blkid + 1], per = (to - from + WPA - 1) / WPA;
                    const int lo = min(to, from + warp * per), hi = min(to, lo + per);
                    if constexpr (RV == 0)
                        leg_run_runs(s, tl, lo, hi, lane, body);
                    else
                        leg_run_conv(s, tl, lo, hi, lane, body);
                }
                group_sync<WPA>();
            }
    }

    /* virial of atom i's energy: every neighbour force times its displacement */
    for (int t = tid; t < n; t += NT) {
        const double4 d = leg_vec(s.d, t);
        const double fx = s.Fnb[3 * t], fy = s.Fnb[3 * t + 1], fz = s.Fnb[3 * t + 2];
        vr[0] += fx * d.x; vr[1] += fy * d.y; vr[2] += fz * d.z;
        vr[3] += fx * d.y; vr[4] += fy * d.z; vr[5] += fz * d.x;
    }
    {
        /* the atom's force and virial: warp sums, then the warps in a fixed order */
        double v[9] = {fi[0], fi[1], fi[2], vr[0], vr[1], vr[2], vr[3], vr[4], vr[5]};
#pragma unroll
        for (int k = 0; k < 9; k++) v[k] = warp_sum(v[k]);
        if (WPA > 1) {
            if (lane == 0)
                for (int k = 0; k < 9; k++) s.red[warp * 9 + k] = v[k];
            group_sync<WPA>();
            if (tid == 0)
                for (int k = 0; k < 9; k++) {
                    double t = 0.0;
                    for (int w = 0; w < WPA; w++) t += s.red[w * 9 + k];
                    v[k] = t;
                }
        }
        if (tid == 0) {
            atomicAdd(&A.F[3 * i], v[0]);
            atomicAdd(&A.F[3 * i + 1], v[1]);
            atomicAdd(&A.F[3 * i + 2], v[2]);
            for (int k = 0; k < 6; k++) A.vir[(size_t)i * 6 + k] = v[3 + k];
        }
        for (int t = tid; t < n; t += NT) {
            const int j = s.j[t];
            atomicAdd(&A.F[3 * j], s.Fnb[3 * t]);
            atomicAdd(&A.F[3 * j + 1], s.Fnb[3 * t + 1]);
            atomicAdd(&A.F[3 * j + 2], s.Fnb[3 * t + 2]);
        }
    }
}

/* ------------------------------------------------------------------ */
/* forward-mode derivative of the descriptors                           */
/* ------------------------------------------------------------------ */

/* dG = (dG/dx) . dx for a displacement field dx[3N] of the atoms and a
 * homogeneous deformation eps[3][3] of every neighbour displacement
 * (d -> d + eps d): the tangent of the descriptor map that the reference
 * materialises as the derivative blocks Fn (dG_j/dx_i) and Sn (dG/dstrain)
 * of PRS_BP (src/nprs.c:567-770), with the same species-0 derivative
 * parameters.  A unit dx on atom m and axis q gives column q of every
 * Fn block of m; eps = e_a e_b^T gives the (a, b) strain column.
 * One warp per atom (one per CTA); every term is added to the atom's
 * descriptor row in shared memory. */
struct JvpArgs {
    int N, cap;
    const int *nn, *nj;
    const double4 *nd;
    const int *spc;
    const mb_params *params;
    const double *dx;
    double eps[9];
    double *dG;
};

__global__ void __launch_bounds__(32) k_jvp(JvpArgs A) {
    extern __shared__ __align__(16) char jsm[];
    const int i = blockIdx.x, lane = threadIdx.x;
    if (i >= A.N) return;
    const mb_params &P = *A.params;
    const int D = P.D, ns = P.nspc, ng2 = P.ng2, cap = A.cap;
    double4 *d = reinterpret_cast<double4 *>(jsm);
    double *dd = reinterpret_cast<double *>(d + cap); /* [cap][3] tangent of each displacement */
    double *g = dd + 3 * cap;                         /* [D] */
    int *rel = reinterpret_cast<int *>(g + D);        /* [cap] relative species */
    const int n = A.nn[i], s0 = A.spc[i];
    for (int t = lane; t < D; t += 32) g[t] = 0.0;
    for (int t = lane; t < n; t += 32) {
        const size_t o = (size_t)i * cap + t;
        const int j = A.nj[o];
        const double4 v = A.nd[o];
        d[t] = v;
        rel[t] = (A.spc[j] - s0 + ns) % ns;
        const double e[3] = {A.eps[0] * v.x + A.eps[1] * v.y + A.eps[2] * v.z,
                             A.eps[3] * v.x + A.eps[4] * v.y + A.eps[5] * v.z,
                             A.eps[6] * v.x + A.eps[7] * v.y + A.eps[8] * v.z};
        for (int q = 0; q < 3; q++) dd[3 * t + q] = A.dx[3 * j + q] - A.dx[3 * i + q] + e[q];
    }
    __syncwarp();
    /* G2: d/dr [fc(r) exp(-eta (r - rs)^2)] dr, dr = d . dd / r */
    for (int t = lane; t < n; t += 32) {
        const double4 v = d[t];
        const double r = v.w, dr = (v.x * dd[3 * t] + v.y * dd[3 * t + 1] + v.z * dd[3 * t + 2]) / r;
        double f2, df2;
        fcut_d(P.d_rc2, r, f2, df2);
        double *gg = g + P.ind2[rel[t]];
        for (int f = 0; f < ng2; f++) {
            const double x = r - P.d_rs[f], eta = P.d_eta2[f];
            atomicAdd(gg + f, exp(-eta * x * x) * (-2.0 * eta * x * f2 + df2) * dr);
        }
    }
    /* G4 over the pairs a < b of the list (the reference's triplets) */
    const int ne = P.ne, nzl = P.nzl;
    for (int a = 0; a + 1 < n; a++) {
        const double4 d1 = d[a];
        const double r1 = d1.w;
        if (!(r1 < P.d_rc4)) continue;
        const double e1x = dd[3 * a], e1y = dd[3 * a + 1], e1z = dd[3 * a + 2];
        const double dr1 = (d1.x * e1x + d1.y * e1y + d1.z * e1z) / r1;
        double f1, df1;
        fcut_d(P.d_rc4, r1, f1, df1);
        for (int b = a + 1 + lane; b < n; b += 32) {
            const double4 d2 = d[b];
            const double r2 = d2.w;
            const double wx = d2.x - d1.x, wy = d2.y - d1.y, wz = d2.z - d1.z;
            const double r3s = wx * wx + wy * wy + wz * wz;
            if (!(r2 < P.d_rc4 && r3s < P.d_rc4sq)) continue;
            const double r3 = sqrt(r3s);
            const double e2x = dd[3 * b], e2y = dd[3 * b + 1], e2z = dd[3 * b + 2];
            const double dr2 = (d2.x * e2x + d2.y * e2y + d2.z * e2z) / r2;
            const double dr3 = (wx * (e2x - e1x) + wy * (e2y - e1y) + wz * (e2z - e1z)) / r3;
            const double c = (d1.x * d2.x + d1.y * d2.y + d1.z * d2.z) / (r1 * r2);
            const double dc = (e1x * d2.x + e1y * d2.y + e1z * d2.z + d1.x * e2x + d1.y * e2y + d1.z * e2z) / (r1 * r2) -
                              c * (dr1 / r1 + dr2 / r2);
            double f2, df2, f3, df3;
            fcut_d(P.d_rc4, r2, f2, df2);
            fcut_d(P.d_rc4, r3, f3, df3);
            const double Af = 2.0 * f1 * f2 * f3;
            const double dA = 2.0 * (df1 * dr1 * f2 * f3 + f1 * df2 * dr2 * f3 + f1 * f2 * df3 * dr3);
            const double rr = r1 * r1 + r2 * r2 + r3s, drr = r1 * dr1 + r2 * dr2 + r3 * dr3;
            double sv[MB_MAXE], tv[MB_MAXE];
            for (int e = 0; e < ne; e++) {
                const double eta = P.d_eta4[e], E = exp(-eta * rr);
                sv[e] = dA * E + Af * E * (-2.0 * eta * drr);
                tv[e] = Af * E * dc;
            }
            double lz[MB_MAXZL], lzp[MB_MAXZL];
            for (int k = 0; k < MB_MAXZL; k++) lz[k] = lzp[k] = 0.0;
            angular<8, 4>(P, c, lz, lzp);
            /* angular<8, 4> lays (zeta, lambda) out as z * 4 + l */
            const int va = rel[a], vb = rel[b];
            const int lo = va < vb ? va : vb, hi = va < vb ? vb : va;
            double *gg = g + P.ind4[lo * lo + hi * hi];
            for (int f = 0; f < P.ng4; f++) {
                const int e = P.g4_e[f], zl = (P.g4_zl[f] / P.nlam) * 4 + P.g4_zl[f] % P.nlam;
                atomicAdd(gg + f, sv[e] * lz[zl] + tv[e] * lzp[zl]);
            }
        }
    }
    (void)nzl;
    __syncwarp();
    for (int t = lane; t < D; t += 32) A.dG[(size_t)i * D + t] = g[t];
}

/* ------------------------------------------------------------------ */
/* reductions                                                          */
/* ------------------------------------------------------------------ */

/* Atoms per CTA of the multi-CTA reductions: chunks of at least 512 atoms,
 * at most MB_RED_MAXB CTAs; nparts = 0 runs one CTA over all atoms. */
__host__ __device__ inline int red_chunk(int N, int nparts) {
    if (nparts <= 0) return N > 0 ? N : 1;
    const int c = (N + MB_RED_MAXB - 1) / MB_RED_MAXB;
    return c > 512 ? c : 512;
}

/* Sum of acc[0..K-1] over the CTA's 256 threads (fixed tree) into red[k][0]. */
template <int K>
__device__ __forceinline__ void block_tree(double (*red)[256], const double *acc, int t) {
    for (int k = 0; k < K; k++) red[k][t] = acc[k];
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (t < h)
            for (int k = 0; k < K; k++) red[k][t] += red[k][t + h];
        __syncthreads();
    }
}

/* After block_tree: CTA partials go to part[cta][0..K-1]; returns true in
 * thread 0 of the CTA that finished last, which then holds the sums of the
 * partials in CTA order in tot[] (and has reset the ticket). */
template <int K>
__device__ __forceinline__ bool last_cta(double (*red)[256], double *part, unsigned *ticket, double *tot, int t) {
    __shared__ bool is_last;
    const int nb = gridDim.x;
    if (nb == 1) {
        if (t == 0)
            for (int k = 0; k < K; k++) tot[k] = red[k][0];
        return t == 0;
    }
    if (t == 0) {
        for (int k = 0; k < K; k++) part[blockIdx.x * 8 + k] = red[k][0];
        __threadfence();
        is_last = atomicAdd(ticket, 1u) == (unsigned)(nb - 1);
    }
    __syncthreads();
    if (!is_last || t != 0) return false;
    __threadfence();
    const volatile double *vp = part;
    for (int k = 0; k < K; k++) {
        double s = 0.0;
        for (int c = 0; c < nb; c++) s += vp[c * 8 + k];
        tot[k] = s;
    }
    *ticket = 0u;
    return true;
}

/* out[0]=E, out[1]=H, out[2..7]=U: every CTA reduces a fixed chunk of atoms
 * (threads strided, then a tree) and zeroes the chunk's force components
 * below 1e-8 (src/cmod.c:177-184); the last CTA adds the partials in CTA
 * order.  Every sum has a fixed order, so results are reproducible. */
__global__ void __launch_bounds__(256) k_finalize(int N, int mode, double pV, const double *EA, const double *EU,
                                                  const double *vir, double *F, double *out, double *part,
                                                  unsigned *ticket) {
    __shared__ double red[7][256];
    const int t = threadIdx.x, chunk = red_chunk(N, part ? 1 : 0);
    const int lo = blockIdx.x * chunk, hi = min(N, lo + chunk);
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int i = lo + t; i < hi; i += 256) {
        acc[0] += EA[i] + EU[i];
        if (mode != MB_MODE_ENERGY)
            for (int k = 0; k < 6; k++) acc[1 + k] += vir[(size_t)i * 6 + k];
    }
    if (mode == MB_MODE_EFS)
        for (int i = 3 * lo + t; i < 3 * hi; i += 256)
            if (fabs(F[i]) < 1e-8) F[i] = 0.0;
    block_tree<7>(red, acc, t);
    double tot[7];
    if (last_cta<7>(red, part, ticket, tot, t)) {
        out[0] = tot[0];
        out[1] = tot[0] + pV;
        for (int k = 0; k < 6; k++) {
            double u = tot[1 + k];
            if (mode == MB_MODE_EFS && fabs(u) < 1e-8) u = 0.0;
            out[2 + k] = u;
        }
    }
}

/* ------------------------------------------------------------------ */
/* NVT step (src/cmod.c:403-407, 440-453)                              */
/* ------------------------------------------------------------------ */

/* K = 1/2 sum m v^2 (CTA chunks, then the partials in CTA order), then
 * xi += dt/tau^2 (2K/(3NT) - 1).  out[8] = K, out[9] = xi;
 * trace[2*step] = H, trace[2*step+1] = K with the step index kept in
 * out[10] and advanced here, so that a captured chunk of steps can be
 * replayed unchanged. */
__global__ void __launch_bounds__(256) k_nvt_thermostat(int N, const double *V, const int *spc, const double *mass,
                                                        double dt, double tau, double T, double *out, double *trace,
                                                        int capTrace, double *part, unsigned *ticket) {
    __shared__ double red[1][256];
    const int t = threadIdx.x, chunk = red_chunk(N, part ? 1 : 0);
    const int lo = blockIdx.x * chunk, hi = min(N, lo + chunk);
    double k[1] = {0.0};
    for (int i = lo + t; i < hi; i += 256) {
        double m = mass[spc[i]];
        k[0] += m * V[3 * i] * V[3 * i] + m * V[3 * i + 1] * V[3 * i + 1] + m * V[3 * i + 2] * V[3 * i + 2];
    }
    block_tree<1>(red, k, t);
    double tot[1];
    if (last_cta<1>(red, part, ticket, tot, t)) {
        double K = 0.5 * tot[0];
        double fs = 1.0 / (tau * tau) * (2.0 * K / ((3.0 * (double)N) * T) - 1.0);
        const int step = (int)out[10];
        out[8] = K;
        out[9] += dt * fs;
        out[10] = (double)(step + 1);
        if (step >= 0 && step < capTrace) {
            trace[2 * step] = out[1];
            trace[2 * step + 1] = K;
        }
    }
}

/* the integrator, then (wrap != 0) the step's closing JAR on the moved
 * atom, the same operations as k_wrap in one launch */
__global__ void k_nvt_integrate(int N, double *X, double *V, const double *F, const int *spc, const double *mass,
                                double dt, const double *out, mb_cell c, int wrap, int *status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double xi = out[9], m = mass[spc[i]];
    for (int q = 0; q < 3; q++) {
        double v = V[3 * i + q];
        double f = F[3 * i + q] / m - xi * v;
        X[3 * i + q] += v * dt + 0.5 * f * dt * dt;
        V[3 * i + q] = v + f * dt;
    }
    if (wrap) wrap_atom(i, X, c, status);
}

__global__ void k_set_out(double *out, int idx, double v) { out[idx] = v; }

} /* namespace */

/* ------------------------------------------------------------------ */
/* launchers                                                           */
/* ------------------------------------------------------------------ */

/* Shapes of the fused kernel: warps per atom x atoms per block.  One warp
 * per atom keeps many atoms resident per SM (large structures); several
 * warps per atom shorten the latency of small structures. */
struct EfsShape {
    int wpa, apb;
};
static const EfsShape kShapes[] = {{1, 4}, {4, 1}, {8, 1}};
#define EFS_STATIC_SMEM (sizeof(mb_params) + 16) /* k_efs's __shared__ Ps, with alignment slack */
#define LEG_STATIC_SMEM (MB_MAXG4 + 16)          /* k_efs_leg's __shared__ g4cell */
#define MB_NSHAPES 3
#define MB_MAX_DEVICES_K 64

/* specialised kernel for the reference bases: 7 G4 exponents, 4 zeta, 2 lambda */
static bool efs_fast(const mb_model *m) { return m->P.ne <= 7 && m->P.nz <= 4 && m->P.nlam <= 2; }

/* triplet-list entries per atom group: all candidate pairs when they fit,
 * otherwise at least one row (the capacity) per warp plus slack */
static int tl_entries(int capNB, int wpa) {
    int all = capNB * (capNB - 1) / 2 + 32 * wpa;
    int lim = wpa == 1 ? 2048 : 8192;
    int floor_ = wpa * (capNB + 64);
    int v = all < lim ? all : lim;
    return v > floor_ ? v : floor_;
}

static size_t group_bytes(const mb_model *m, int capNB, int wpa) {
    bool fast = efs_fast(m);
    int ne = fast ? 7 : MB_MAXE;
    int cells = fast ? 7 * 8 : MB_MAXE * 8 * 4;
    return (efs_smem_bytes(capNB, m->P.D, ne, m->P.ng2, cells, wpa, tl_entries(capNB, wpa), fast ? 1 : 0) + 15) &
           ~(size_t)15;
}

extern "C" size_t mbk_efs_smem(const mb_model *m, int capNB, int shape) {
    return group_bytes(m, capNB, kShapes[shape].wpa) * kShapes[shape].apb;
}

extern "C" int mbk_wrap(mb_dev *d, int N, const mb_cell *c, void *stream, long *launches) {
    if (c->ND <= 0 || N <= 0) return 0;
    k_wrap<<<(N + 127) / 128, 128, 0, (cudaStream_t)stream>>>(N, d->X, *c, d->status);
    (*launches)++;
    return (int)cudaGetLastError();
}

extern "C" int mbk_nlist(mb_dev *d, int N, int NM, const mb_cell *c, double rc, void *stream, long *launches) {
    cudaStream_t st = (cudaStream_t)stream;
    double rc2 = rc * rc;
    int warps_per_block = 4;
    int blocks = (N + warps_per_block - 1) / warps_per_block;
    if (c->M[0] > 0) {
        int ncell = c->M[0] * c->M[1] * c->M[2];
        cudaMemsetAsync(d->cell_cnt, 0, sizeof(int) * ncell, st);
        k_cell_bin<<<(N + 127) / 128, 128, 0, st>>>(N, d->X, *c, d->cell_of, d->cell_cnt);
        k_cell_scan<<<1, 1024, 0, st>>>(ncell, d->cell_cnt, d->cell_start);
        cudaMemsetAsync(d->cell_cnt, 0, sizeof(int) * ncell, st);
        k_cell_fill<<<(N + 127) / 128, 128, 0, st>>>(N, d->cell_of, d->cell_start, d->cell_cnt, d->cell_atoms);
        k_cell_sort<<<(ncell + 3) / 4, 128, 0, st>>>(ncell, d->cell_start, d->cell_atoms); /* a warp per cell */
        k_nlist_cell<<<blocks, warps_per_block * 32, 0, st>>>(N, NM, d->capNB, d->X, *c, rc2, d->cell_of,
                                                              d->cell_start, d->cell_atoms, d->nn, d->nj,
                                                              (double4 *)d->nd, d->status,
                                                              d->legs_on ? d->nk : nullptr);
        *launches += 5;
    } else {
        k_nlist_brute<<<blocks, warps_per_block * 32, 0, st>>>(N, NM, d->capNB, d->X, *c, rc2, d->nn, d->nj,
                                                               (double4 *)d->nd, d->status,
                                                               d->legs_on ? d->nk : nullptr);
        *launches += 1;
    }
    return (int)cudaGetLastError();
}

template <int NE, int NZ, int NLAM, int WPA, int APB>
static int launch_shape(const EfsArgs &a, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1) {
    auto kern = k_efs<NE, NZ, NLAM, WPA, APB>;
    size_t smem = a.smem_group * APB;
    /* the shared-memory opt-in is a per-device attribute of the function:
     * remembered per device */
    static size_t configured[MB_MAX_DEVICES_K] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MB_MAX_DEVICES_K) return (int)cudaErrorInvalidDevice;
    /* the 48 KB default and the 227 KB opt-in limit both count the kernel's
     * static shared block (the staged mb_params) as well as the dynamic part */
    if (smem + EFS_STATIC_SMEM > 227 * 1024) return (int)cudaErrorInvalidConfiguration;
    if (smem + EFS_STATIC_SMEM > 48 * 1024 && smem > configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
        configured[dev] = smem;
    }
    if (e0) mbk_record(e0, st);
    kern<<<(a.N + APB - 1) / APB, WPA * 32 * APB, smem, st>>>(a);
    if (e1) mbk_record(e1, st);
    return (int)cudaGetLastError();
}

static int launch_any(const mb_model *m, int shape, EfsArgs a, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1) {
    a.smem_group = group_bytes(m, a.cap, kShapes[shape].wpa);
    a.tl_cap = tl_entries(a.cap, kShapes[shape].wpa);
    if (efs_fast(m)) {
        switch (shape) {
            case 0: return launch_shape<7, 4, 2, 1, 4>(a, st, e0, e1);
            case 1: return launch_shape<7, 4, 2, 4, 1>(a, st, e0, e1);
            default: return launch_shape<7, 4, 2, 8, 1>(a, st, e0, e1);
        }
    }
    if (m->P.nz > 8 || m->P.nlam > 4) return (int)cudaErrorInvalidValue;
    switch (shape) {
        case 0: return launch_shape<MB_MAXE, 8, 4, 1, 4>(a, st, e0, e1);
        case 1: return launch_shape<MB_MAXE, 8, 4, 4, 1>(a, st, e0, e1);
        default: return launch_shape<MB_MAXE, 8, 4, 8, 1>(a, st, e0, e1);
    }
}

/* ---- leg-table path ---- */

/* The leg-table path applies to the model: every forward and derivative
 * function shares the list cutoff, the pair-mixed G4 exponents equal the
 * species-0 ones to rounding (so one leg row serves the energy and the
 * derivative terms), and the basis has the reference's shape (<= 8 G4
 * exponents, <= 4 integer zeta, <= 2 lambda). */
static bool leg_model_ok(const mb_model *m) {
    const mb_params &P = m->P;
    if (P.ng4 < 1 || P.ne > 8 || P.nz > 4 || P.nlam > 2 || !P.zeta_int) return false;
    const double rc = m->rc_list;
    if (P.d_rc2 != rc || P.d_rc4 != rc) return false;
    for (int s = 0; s < P.nspc; s++)
        for (int t = 0; t < P.nspc; t++) {
            const int p = s * s + t * t;
            if (P.f_rc2[p] != rc || P.f_rc4[p] != rc) return false;
            for (int e = 0; e < P.ne; e++)
                if (fabs(P.f_eta4[p][e] - P.d_eta4[e]) > 1e-12 * fabs(P.d_eta4[e])) return false;
        }
    return true;
}

extern "C" int mbk_legs_model(const mb_model *m) { return leg_model_ok(m) ? 1 : 0; }

/* 1 when a pass of N atoms in cell c can run on leg tables: the model
 * qualifies, the tables are allocated, and every entry key fits (atom
 * index in 17 bits, images within +-15, neighbour capacity <= 128) */
extern "C" int mbk_legs_usable(const mb_dev *d, const mb_model *m, int N, const mb_cell *c) {
    if (!d->nk || !d->leg || !d->nso || !d->trip || !d->tboff || !d->lhash) return 0;
    if (N >= MB_LEG_MAX_ATOMS || d->capNB > MB_LEG_MAX_CAP) return 0;
    for (int q = 0; q < 3; q++)
        if (c->Nq[q] > MB_LEG_MAX_IMAGE) return 0;
    return leg_model_ok(m) ? 1 : 0;
}

/* shapes 0-3 with the per-lane-run reverse layout, 4-7 the same shapes
 * with the consecutive-entry layout */
static const EfsShape kLegShapes[] = {{1, 4}, {1, 2}, {2, 1}, {4, 1}, {1, 4}, {1, 2}, {2, 1}, {4, 1}};
#define MB_NLEGSHAPES 8

static size_t leg_group_bytes(const mb_model *m, int capNB, int wpa) {
    return leg_smem_bytes(capNB, m->P.D, m->P.ng2, wpa);
}

template <int NE, int WPA, int APB, int RV>
static int launch_leg(const LegArgs &a, cudaStream_t st) {
    auto kern = k_efs_leg<NE, WPA, APB, RV>;
    const size_t smem = a.smem_group * APB;
    static size_t configured[MB_MAX_DEVICES_K] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MB_MAX_DEVICES_K) return (int)cudaErrorInvalidDevice;
    if (smem + LEG_STATIC_SMEM > 227 * 1024) return (int)cudaErrorInvalidConfiguration;
    if (smem + LEG_STATIC_SMEM > 48 * 1024 && smem > configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
        configured[dev] = smem;
    }
    kern<<<(a.N + APB - 1) / APB, WPA * 32 * APB, smem, st>>>(a);
    return (int)cudaGetLastError();
}

/* k_legs, k_trip, then k_efs_leg in shape `shape`; the events (if any) bracket the three */
static int launch_leg_pass(const mb_dev *d, const mb_model *m, int shape, LegArgs a, cudaStream_t st, cudaEvent_t e0,
                           cudaEvent_t e1) {
    a.smem_group = leg_group_bytes(m, a.cap, kLegShapes[shape].wpa);
    if (e0) mbk_record(e0, st);
    k_legs<<<(a.N + 3) / 4, 128, 0, st>>>(a.N, a.cap, d->nn, d->nj, d->nk, (double4 *)d->nd, d->spc, d->params,
                                         d->leg, d->nso, (uint2 *)d->lhash);
    k_trip<<<(a.N + TRIP_WARPS - 1) / TRIP_WARPS, 32 * TRIP_WARPS, 0, st>>>(
        a.N, a.cap, d->tcap, m->P.nspc, d->nn, d->nj, d->nk, (const double4 *)d->nd, d->nso, d->spc, d->params,
        (const uint2 *)d->lhash, (uint2 *)d->trip, d->tboff, a.counters);
    int rc;
    if (m->P.ne <= 7) {
        switch (shape) {
            case 0: rc = launch_leg<7, 1, 4, 0>(a, st); break;
            case 1: rc = launch_leg<7, 1, 2, 0>(a, st); break;
            case 2: rc = launch_leg<7, 2, 1, 0>(a, st); break;
            case 3: rc = launch_leg<7, 4, 1, 0>(a, st); break;
            case 4: rc = launch_leg<7, 1, 4, 1>(a, st); break;
            case 5: rc = launch_leg<7, 1, 2, 1>(a, st); break;
            case 6: rc = launch_leg<7, 2, 1, 1>(a, st); break;
            default: rc = launch_leg<7, 4, 1, 1>(a, st); break;
        }
    } else {
        switch (shape) {
            case 0: rc = launch_leg<8, 1, 4, 0>(a, st); break;
            case 1: rc = launch_leg<8, 1, 2, 0>(a, st); break;
            case 2: rc = launch_leg<8, 2, 1, 0>(a, st); break;
            case 3: rc = launch_leg<8, 4, 1, 0>(a, st); break;
            case 4: rc = launch_leg<8, 1, 4, 1>(a, st); break;
            case 5: rc = launch_leg<8, 1, 2, 1>(a, st); break;
            case 6: rc = launch_leg<8, 2, 1, 1>(a, st); break;
            default: rc = launch_leg<8, 4, 1, 1>(a, st); break;
        }
    }
    if (e1) mbk_record(e1, st);
    return rc;
}

/* warps per atom and atoms per CTA of shape `shape` of the leg kernel
 * (legs != 0) or of k_efs */
extern "C" int mbk_shape_dims(int legs, int shape, int *wpa, int *apb) {
    if (shape < 0 || shape >= (legs ? MB_NLEGSHAPES : MB_NSHAPES)) return 1;
    const EfsShape &e = legs ? kLegShapes[shape] : kShapes[shape];
    *wpa = e.wpa;
    *apb = e.apb;
    return 0;
}

/* Autotuner: on the first pass of a (mode, size bucket, capacity) the three
 * shapes are each timed once (after an untimed launch) and the fastest is
 * kept for later passes of that key. */
static int tune_key(const mb_dev *d, int N, int mode) {
    int bucket = 0;
    while ((1 << bucket) < N) bucket++;
    return (mode << 28) | ((d->legs_on ? 1 : 0) << 26) | (bucket << 20) | (d->capNB & 0xfffff);
}

/* Decision for a pass that may run on leg tables: the four leg shapes and
 * the shapes of k_efs are each timed once (after an untimed launch) and the
 * fastest kept, 16 + shape for the leg path, shape for k_efs.  Small
 * structures (a few dozen atoms: one CTA per atom, most SMs idle) can favour
 * k_efs's many-warp shapes; large ones the leg path. */
static int tune_family(mb_dev *d, const mb_model *m, int N, int mode, const LegArgs &la, const EfsArgs &a,
                       cudaStream_t st) {
    const int key = tune_key(d, N, mode);
    for (int k = 0; k < d->tune_n; k++)
        if (d->tune_key[k] == key) return d->tune_val[k];
    int best = 16;
    if (d->tune_fixed >= 0) {
        /* a forced shape (of the leg path) is recorded as the decision for this key */
        best = 16 + (d->tune_fixed < MB_NLEGSHAPES ? d->tune_fixed : 0);
    } else {
        LegArgs tl = la;
        EfsArgs te = a;
        tl.counters = nullptr;
        te.counters = nullptr;
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        float best_ms = 1e30f;
        for (int c = 0; c < MB_NLEGSHAPES + MB_NSHAPES; c++) {
            const bool leg = c < MB_NLEGSHAPES;
            const int sh = leg ? c : c - MB_NLEGSHAPES;
            const size_t need = leg ? leg_group_bytes(m, la.cap, kLegShapes[sh].wpa) * kLegShapes[sh].apb + LEG_STATIC_SMEM
                                    : group_bytes(m, a.cap, kShapes[sh].wpa) * kShapes[sh].apb + EFS_STATIC_SMEM;
            if (need > 227 * 1024) continue;
            float ms = 1e30f;
            int bad = 0;
            for (int rep = 0; rep < 2 && !bad; rep++) {
                if (mode == MB_MODE_EFS || mode == MB_MODE_VJP) cudaMemsetAsync(d->F, 0, sizeof(double) * 3 * N, st);
                bad = leg ? launch_leg_pass(d, m, sh, tl, st, rep ? e0 : nullptr, rep ? e1 : nullptr)
                          : launch_any(m, sh, te, st, rep ? e0 : nullptr, rep ? e1 : nullptr);
            }
            if (!bad && cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best_ms) {
                best_ms = ms;
                best = leg ? 16 + sh : sh;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaGetLastError();
    }
    if (d->tune_n < MB_TUNE_SLOTS) {
        d->tune_key[d->tune_n] = key;
        d->tune_val[d->tune_n] = best;
        d->tune_n++;
    }
    return best;
}

static int tune_shape(mb_dev *d, const mb_model *m, int N, int mode, const EfsArgs &a, cudaStream_t st) {
    int k;
    const int key = tune_key(d, N, mode);
    for (k = 0; k < d->tune_n; k++)
        if (d->tune_key[k] == key) return d->tune_val[k];
    if (d->tune_fixed >= 0) {
        const int v = d->tune_fixed < MB_NSHAPES ? d->tune_fixed : 0;
        if (d->tune_n < MB_TUNE_SLOTS) {
            d->tune_key[d->tune_n] = key;
            d->tune_val[d->tune_n++] = v;
        }
        return v;
    }
    EfsArgs t = a;
    t.counters = nullptr;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int best = 0;
    float best_ms = 1e30f;
    for (int sh = 0; sh < MB_NSHAPES; sh++) {
        if (group_bytes(m, a.cap, kShapes[sh].wpa) * kShapes[sh].apb + EFS_STATIC_SMEM > 227 * 1024) continue;
        float ms = 1e30f;
        for (int rep = 0; rep < 2; rep++) {
            if (mode == MB_MODE_EFS || mode == MB_MODE_VJP) cudaMemsetAsync(d->F, 0, sizeof(double) * 3 * N, st);
            if (launch_any(m, sh, t, st, rep ? e0 : nullptr, rep ? e1 : nullptr)) break;
        }
        if (cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) {
            best_ms = ms;
            best = sh;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaGetLastError();
    if (d->tune_n < MB_TUNE_SLOTS) {
        d->tune_key[d->tune_n] = key;
        d->tune_val[d->tune_n] = best;
        d->tune_n++;
    }
    return best;
}

extern "C" int mbk_descriptor_pass(mb_dev *d, const mb_model *m, int N, int mode, double urep, int need_nb_max,
                                   int nb_max, void *stream, long *launches) {
    (void)need_nb_max;
    (void)nb_max;
    cudaStream_t st = (cudaStream_t)stream;
    EfsArgs a;
    a.N = N;
    a.cap = d->capNB;
    a.mode = mode;
    a.urep = urep;
    a.nn = d->nn;
    a.nj = d->nj;
    a.nd = (const double4 *)d->nd;
    a.spc = d->spc;
    a.params = d->params;
    a.weights = d->weights;
    a.EA = d->EA;
    a.EU = d->EU;
    a.G = d->G;
    a.F = d->F;
    a.vir = d->vir;
    a.counters = d->counters;
    a.smem_group = 0;
    cudaMemsetAsync(d->EU, 0, sizeof(double) * N, st);
    int fam = -1; /* k_efs shape chosen against the leg path */
    if (d->legs_on) {
        LegArgs la;
        la.N = N;
        la.cap = d->capNB;
        la.mode = mode;
        la.urep = urep;
        la.nn = d->nn;
        la.nj = d->nj;
        la.nso = d->nso;
        la.nd = (const double4 *)d->nd;
        la.trip = (const uint2 *)d->trip;
        la.tboff = d->tboff;
        la.tcap = d->tcap;
        la.leg = d->leg;
        la.spc = d->spc;
        la.params = d->params;
        la.weights = d->weights;
        la.EA = d->EA;
        la.EU = d->EU;
        la.G = d->G;
        la.F = d->F;
        la.vir = d->vir;
        la.counters = d->counters;
        la.smem_group = 0;
        la.P = m->P;
        const int v = tune_family(d, m, N, mode, la, a, st);
        if (v >= 16) {
            d->last_shape = v;
            cudaEvent_t e0 = 0, e1 = 0;
            if (d->ev_on && d->ev_n < d->ev_cap) {
                e0 = ((cudaEvent_t *)d->ev_pool)[2 * d->ev_n];
                e1 = ((cudaEvent_t *)d->ev_pool)[2 * d->ev_n + 1];
                d->ev_n++;
            }
            if (mode == MB_MODE_EFS || mode == MB_MODE_VJP) cudaMemsetAsync(d->F, 0, sizeof(double) * 3 * N, st);
            const int rc = launch_leg_pass(d, m, v - 16, la, st, e0, e1);
            (*launches) += 3;
            return rc;
        }
        fam = v;
    }
    int shape = fam >= 0 ? fam : tune_shape(d, m, N, mode, a, st);
    d->last_shape = shape;
    cudaEvent_t e0 = 0, e1 = 0;
    if (d->ev_on && d->ev_n < d->ev_cap) {
        e0 = ((cudaEvent_t *)d->ev_pool)[2 * d->ev_n];
        e1 = ((cudaEvent_t *)d->ev_pool)[2 * d->ev_n + 1];
        d->ev_n++;
    }
    if (mode == MB_MODE_EFS || mode == MB_MODE_VJP) cudaMemsetAsync(d->F, 0, sizeof(double) * 3 * N, st);
    int rc = launch_any(m, shape, a, st, e0, e1);
    (*launches)++;
    return rc;
}

/* the descriptor tangent for displacements dx[3N] (device) and the
 * deformation eps[9] (host), into dG[N*D] (device) */
extern "C" int mbk_jvp(mb_dev *d, const mb_model *m, int N, const double *dx, const double *eps, double *dG,
                       void *stream, long *launches) {
    if (m->P.nz > 8 || m->P.nlam > 4) return (int)cudaErrorInvalidValue;
    JvpArgs a;
    a.N = N;
    a.cap = d->capNB;
    a.nn = d->nn;
    a.nj = d->nj;
    a.nd = (const double4 *)d->nd;
    a.spc = d->spc;
    a.params = d->params;
    a.dx = dx;
    for (int k = 0; k < 9; k++) a.eps[k] = eps ? eps[k] : 0.0;
    a.dG = dG;
    const size_t smem = sizeof(double4) * d->capNB + sizeof(double) * (3 * (size_t)d->capNB + m->P.D) +
                        sizeof(int) * d->capNB;
    if (smem > 227 * 1024) return (int)cudaErrorInvalidConfiguration;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_jvp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
    }
    k_jvp<<<N, 32, smem, (cudaStream_t)stream>>>(a);
    (*launches)++;
    return (int)cudaGetLastError();
}

extern "C" int mbk_finalize(mb_dev *d, int N, int mode, double pV, void *stream, long *launches) {
    const int chunk = red_chunk(N, d->part ? 1 : 0), nb = (N + chunk - 1) / chunk;
    k_finalize<<<nb > 0 ? nb : 1, 256, 0, (cudaStream_t)stream>>>(N, mode, pV, d->EA, d->EU, d->vir, d->F, d->out,
                                                                   d->part, d->ticket);
    (*launches)++;
    return (int)cudaGetLastError();
}

extern "C" int mbk_nvt_update(mb_dev *d, const mb_model *m, int N, double dt, double tau, double T,
                              const mb_cell *c, void *stream, long *launches) {
    cudaStream_t st = (cudaStream_t)stream;
    (void)m;
    /* masses by species live after the weights in the parameter upload (see mb_core.c) */
    const double *mass = d->weights + m->weights_len;
    const int chunk = red_chunk(N, d->part ? 1 : 0), nb = (N + chunk - 1) / chunk;
    k_nvt_thermostat<<<nb > 0 ? nb : 1, 256, 0, st>>>(N, d->V, d->spc, mass, dt, tau, T, d->out, d->trace,
                                                      d->capTrace, d->part ? d->part + MB_RED_MAXB * 8 : nullptr,
                                                      d->ticket ? d->ticket + 1 : nullptr);
    k_nvt_integrate<<<(N + 127) / 128, 128, 0, st>>>(N, d->X, d->V, d->F, d->spc, mass, dt, d->out, *c,
                                                     c->ND > 0 ? 1 : 0, d->status);
    *launches += 2;
    return (int)cudaGetLastError();
}

extern "C" int mbk_set_out(mb_dev *d, int idx, double v, void *stream) {
    k_set_out<<<1, 1, 0, (cudaStream_t)stream>>>(d->out, idx, v);
    return (int)cudaGetLastError();
}

/* events recorded while the stream is being captured become event-record
 * nodes of the graph, so that they time every replay */
extern "C" void mbk_record(void *event, void *stream) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing((cudaStream_t)stream, &cs);
    if (cs == cudaStreamCaptureStatusActive)
        cudaEventRecordWithFlags((cudaEvent_t)event, (cudaStream_t)stream, cudaEventRecordExternal);
    else
        cudaEventRecord((cudaEvent_t)event, (cudaStream_t)stream);
}

/* 1 when the descriptor pass of (N, mode) at the current capacity has its
 * kernel shape already: only then may it be captured (tuning synchronises) */
extern "C" int mbk_shape_ready(const mb_dev *d, int N, int mode) {
    int k;
    if (d->tune_fixed >= 0) return 1;
    const int key = tune_key(d, N, mode);
    for (k = 0; k < d->tune_n; k++)
        if (d->tune_key[k] == key) return 1;
    return 0;
}

/* ------------------------------------------------------------------ */
/* Replayed single-structure passes: the kernel nodes of a captured     */
/* pass that take the cell (or pV) by value, and their update          */
/* ------------------------------------------------------------------ */

template <typename... A>
constexpr int karity(void (*)(A...)) {
    return (int)sizeof...(A);
}

struct CellArg {
    const void *func;
    int arity, index; /* index of the mb_cell argument; -1: the pV argument of k_finalize */
};

static const CellArg kCellArgs[] = {
    {(const void *)k_wrap, karity(k_wrap), 2},
    {(const void *)k_cell_bin, karity(k_cell_bin), 2},
    {(const void *)k_nlist_cell, karity(k_nlist_cell), 4},
    {(const void *)k_nlist_brute, karity(k_nlist_brute), 4},
    {(const void *)k_finalize, karity(k_finalize), -1},
};

/* Find in `graph` the kernel nodes whose arguments depend on the cell or
 * pV; stores up to `cap` of them (node, table row) and returns how many
 * there are, or -1 on an error. */
extern "C" int mbk_graph_cell_nodes(void *graph, void **nodes, int *rows, int cap) {
    size_t n = 0;
    if (cudaGraphGetNodes((cudaGraph_t)graph, nullptr, &n) != cudaSuccess) return -1;
    cudaGraphNode_t *all = (cudaGraphNode_t *)malloc(sizeof(cudaGraphNode_t) * (n ? n : 1));
    if (cudaGraphGetNodes((cudaGraph_t)graph, all, &n) != cudaSuccess) {
        free(all);
        return -1;
    }
    int found = 0;
    for (size_t k = 0; k < n; k++) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(all[k], &t) != cudaSuccess || t != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams kp;
        if (cudaGraphKernelNodeGetParams(all[k], &kp) != cudaSuccess) continue;
        for (int r = 0; r < (int)(sizeof(kCellArgs) / sizeof(kCellArgs[0])); r++)
            if (kp.func == kCellArgs[r].func) {
                if (found < cap) {
                    nodes[found] = (void *)all[k];
                    rows[found] = r;
                }
                found++;
            }
    }
    free(all);
    return found;
}

/* Point the recorded nodes of the instantiated graph at a new cell and pV. */
extern "C" int mbk_graph_set_cell(void *exec, void *const *nodes, const int *rows, int count, const mb_cell *c,
                                  double pV) {
    for (int k = 0; k < count; k++) {
        cudaKernelNodeParams kp;
        cudaError_t e = cudaGraphKernelNodeGetParams((cudaGraphNode_t)nodes[k], &kp);
        if (e != cudaSuccess) return (int)e;
        const CellArg &a = kCellArgs[rows[k]];
        void *args[16];
        if (a.arity > 16) return (int)cudaErrorInvalidValue;
        for (int q = 0; q < a.arity; q++) args[q] = kp.kernelParams[q];
        mb_cell cell = *c;
        double pv = pV;
        if (a.index >= 0)
            args[a.index] = &cell;
        else
            args[2] = &pv;
        kp.kernelParams = args;
        kp.extra = nullptr;
        e = cudaGraphExecKernelNodeSetParams((cudaGraphExec_t)exec, (cudaGraphNode_t)nodes[k], &kp);
        if (e != cudaSuccess) return (int)e;
    }
    return 0;
}
