/*
 * mb_batch.cu -- relaxation of a population of small structures in one
 * persistent launch (the batched counterpart of RELX_INT's serial loop,
 * src/emod.c:521-548).
 *
 * Each CTA takes structures from an atomic work counter and relaxes each
 * one completely on the device:
 *   - BFGS over the DOF vector of CELL_MIN (fractional coordinates, then
 *     the nine lattice components, src/cmin.c:22-88), FP64 state: the
 *     inverse Hessian in per-CTA global scratch, the vectors in shared
 *     memory; Fletcher's line search (Algorithms 2.6.2/2.6.4) driven by
 *     thread 0 with the CTA evaluating every trial point;
 *   - each evaluation: wrap, brute-force periodic neighbour list (FP64
 *     displacements), and per atom (one warp each) the G2/G4 descriptors,
 *     MLP and reverse pass in FP32, with forces gathered in shared memory and
 *     energy and virial reduced in FP64; the repulsion term in FP64;
 *   - the gradient of cdfunc_gsl (src/cmin.c:107-166) in FP64.
 * A structure stops when max |F| < fmax and max |U - pV| / N < fmax.
 */
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdlib.h>
#include <math_constants.h>
#include <stdint.h>

#include "../../../include/maise_b200.h"
#include "../mb_internal.h"

#define FULLM 0xffffffffu

namespace {

constexpr int BMAXN = 64;
constexpr int BMAXNB = 96;
constexpr int BMAXDOF = 3 * BMAXN + 9;
constexpr int BMAXD = 288;
constexpr int BTL = 1024;
/* warps per structure: 12 (one structure per SM) by default, 4 (three
 * structures per SM) on request.  Both hold the 12 warps per SM that 168
 * registers a thread allow; the wide CTA finishes each structure in about a
 * third of the time, which bounds a launch through its slowest structure,
 * and runs the per-structure FP64 work (BFGS vectors, list builds) on three
 * times the threads, so it is also the faster one for large populations
 * (20000 Cu-Pd-Ag offspring of 16-48 atoms: 9.7 s against 14.9 s) */
constexpr int BWARPS_WIDE = 12;
constexpr int BIMG = 4; /* image shifts a lane holds in the fast neighbour search (128 images) */
constexpr int BNE = 7, BNZ = 4, BNLAM = 2, BNZL = 8, BCELLS = 64;

/* FP32 copy of the descriptor parameters (fast basis layout only) */
struct BParams {
    int nspc, D, ng2, ng4, ne, nz, nlam, h1, h2;
    int ind2[4], ind4[20];
    float f_rc2[MB_NPAIR], f_rc4[MB_NPAIR], f_rc4sq[MB_NPAIR];
    float f_eta2[MB_NPAIR][MB_MAXG2], f_rs[MB_NPAIR][MB_MAXG2], f_eta4[MB_NPAIR][MB_MAXE];
    float d_rc2, d_rc4, d_rc4sq;
    float d_eta2[MB_MAXG2], d_rs[MB_MAXG2], d_eta4[MB_MAXE];
    float lam[MB_MAXL], powz[MB_MAXZ], zeta[MB_MAXZ];
    int zbits[MB_MAXZ], zm1bits[MB_MAXZ];
    int zstd; /* zeta = {1, 2, 4, 16} in this order */
    int g4_cell[MB_MAXG4];
    double rm[MB_MAXSPC];
    double rc;
    int w_off[MB_MAXSPC];
};

struct BArgs {
    int S, rlxt, mitr;
    double p_ev, urep, fmax, sigma;
    const int *nat, *off, *spc;
    const int *order; /* queue position -> structure (largest first) */
    double *lat, *x, *H;
    int *iters, *status;
    /* optional: forces [3 * atoms] and virial U [6 * S] at each structure's
     * final state (FP32 evaluation, FP64 reductions); NULL to skip */
    double *fout, *uout;
    const BParams *P;
    const float *W;
    int *queue;
    double *hmat;  /* per CTA: BMAXDOF^2 */
    float4 *nbd;   /* per CTA: BMAXN * BMAXNB */
    int *nbj;      /* per CTA: BMAXN * BMAXNB */
    long long *evals;
    /* work done (for the roofline): atom evaluations, neighbour pairs and
     * triplets of the forward pass; per-warp counts added at kernel exit */
    unsigned long long *work;
};

struct WarpWS {
    float4 d[BMAXNB];
    float ir[BMAXNB], fa[BMAXNB], fb[BMAXNB];
    alignas(16) float P[BMAXNB * 8]; /* exp(-eta r^2) per neighbour, BNE used of 8 */
    float Fnb[BMAXNB * 3];
    alignas(16) float grid[BCELLS];
    float G[BMAXD];
    float h[4 * MB_MAXH];
    float red[64];
    int j[BMAXNB], sp[BMAXNB], raw[BMAXNB];
    unsigned tl[BTL];
    int blk[6][2];
    int seg[8];
    unsigned long long work[3]; /* atom evaluations, pairs, triplets of this warp */
};

template <int W>
struct BShared {
    double L[9], R[9];
    double xc[BMAXN * 3];
    double ea[BMAXN], eu[BMAXN];
    double x[BMAXDOF], g[BMAXDOF], p[BMAXDOF], xt[BMAXDOF], gt[BMAXDOF], xa[BMAXDOF], ga[BMAXDOF], hy[BMAXDOF];
    double vir[W][6];
    double uvir[6];
    double red[W * 32];
    double scal[24];
    double F[BMAXN * 3];
    int spc[BMAXN];
    int nn[BMAXN];
    int s, N, ndof, flag, cmd, first;
    /* posted by the cluster's rank 0 before each evaluation: structure
     * (-1: exit) and which DOF vector (0: x, 1: xt) the other ranks copy */
    int cmd_s, cmd_dof;
    WarpWS ws[W];
};

/* ---------------- small helpers ---------------- */

__device__ __forceinline__ float fcutf(float rc, float r) { return r > rc ? 0.0f : 0.5f * (cospif(r / rc) + 1.0f); }

__device__ __forceinline__ void fcutf_d(float rc, float r, float &f, float &df) {
    if (r > rc) {
        f = 0.0f;
        df = 0.0f;
        return;
    }
    float s, c;
    sincospif(r / rc, &s, &c);
    f = 0.5f * (c + 1.0f);
    df = -0.5f * CUDART_PI_F / rc * s;
}

__device__ __forceinline__ void angularf(const BParams &P, float c, float *lz, float *lzp) {
    if (P.zstd) {
        /* zeta = 1, 2, 4, 16: (1 + lam c)^zeta by squaring, and the
         * zeta - 1 = 0, 1, 3, 15 powers of the derivative from the same squares */
#pragma unroll
        for (int l = 0; l < BNLAM; l++) {
            const float lam = P.lam[l], b1 = 1.0f + lam * c, b2 = b1 * b1, b4 = b2 * b2, b8 = b4 * b4;
            const float pw[4] = {b1, b2, b4, b8 * b8};
            const float pm[4] = {1.0f, b1, b2 * b1, b8 * b4 * b2 * b1};
#pragma unroll
            for (int z = 0; z < 4; z++) {
                lz[z * BNLAM + l] = P.powz[z] * pw[z];
                if (lzp) lzp[z * BNLAM + l] = P.powz[z] * P.zeta[z] * lam * pm[z];
            }
        }
        return;
    }
#pragma unroll
    for (int l = 0; l < BNLAM; l++) {
        float lam = P.lam[l], base = 1.0f + lam * c;
        float sq[7];
        sq[0] = base;
#pragma unroll
        for (int k = 1; k < 7; k++) sq[k] = sq[k - 1] * sq[k - 1];
#pragma unroll
        for (int z = 0; z < BNZ; z++) {
            int zb = P.zbits[z], mb = P.zm1bits[z];
            float pw = 1.0f, pm = 1.0f;
#pragma unroll
            for (int k = 0; k < 7; k++) {
                if (zb & (1 << k)) pw *= sq[k];
                if (mb & (1 << k)) pm *= sq[k];
            }
            lz[z * BNLAM + l] = P.powz[z] * pw;
            if (lzp) lzp[z * BNLAM + l] = P.powz[z] * P.zeta[z] * lam * pm;
        }
    }
}

__device__ __forceinline__ double bsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULLM, v, o);
    return v;
}
__device__ __forceinline__ float bsumf(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULLM, v, o);
    return v;
}

/* Sum of 64 per-lane accumulators across the warp by recursive halving: at
 * each step a lane keeps one half of its cells and adds its partner's copy
 * of that half (32 + 16 + 8 + 4 + 2 exchanges).  On return lane l holds the
 * totals of cells 2l and 2l+1 in v[0], v[1]. */
__device__ __forceinline__ void warp_reduce64f(float *v, int lane) {
#pragma unroll
    for (int step = 0; step < 5; step++) {
        const int off = 16 >> step, half = 32 >> step;
        const bool upper = (lane & off) != 0;
#pragma unroll
        for (int k = 0; k < half; k++) {
            const float send = upper ? v[k] : v[k + half];
            const float keep = upper ? v[k + half] : v[k];
            v[k] = keep + __shfl_xor_sync(FULLM, send, off);
        }
    }
}

/* Sum of 16 per-lane accumulators across the warp: four halving steps
 * (8 + 4 + 2 + 1 exchanges) leave lanes l and l^1 with partial sums of cell
 * (l >> 1) & 15, and one more exchange completes it in both. */
__device__ __forceinline__ float warp_reduce16f(float *v, int lane) {
#pragma unroll
    for (int step = 0; step < 4; step++) {
        const int off = 16 >> step, half = 8 >> step;
        const bool upper = (lane & off) != 0;
#pragma unroll
        for (int k = 0; k < half; k++) {
            const float send = upper ? v[k] : v[k + half];
            const float keep = upper ? v[k + half] : v[k];
            v[k] = keep + __shfl_xor_sync(FULLM, send, off);
        }
    }
    return v[0] + __shfl_xor_sync(FULLM, v[0], 1);
}

/* CTA-wide sum of one double per thread (all threads get the result) */
template <int W>
__device__ double cta_sum(BShared<W> &sh, double v) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = bsum(v);
    __syncthreads();
    if (lane == 0) sh.red[w] = v;
    __syncthreads();
    double t = 0.0;
    for (int k = 0; k < W; k++) t += sh.red[k];
    __syncthreads();
    return t;
}

template <int W>
__device__ double cta_max(BShared<W> &sh, double v) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULLM, v, o));
    __syncthreads();
    if (lane == 0) sh.red[w] = v;
    __syncthreads();
    double t = 0.0;
    for (int k = 0; k < W; k++) t = fmax(t, sh.red[k]);
    __syncthreads();
    return t;
}

__device__ void reciprocal9(const double *L, double *R) {
    R[6] = L[1] * L[5] - L[2] * L[4];
    R[7] = L[2] * L[3] - L[0] * L[5];
    R[8] = L[0] * L[4] - L[1] * L[3];
    R[0] = L[4] * L[8] - L[5] * L[7];
    R[1] = L[5] * L[6] - L[3] * L[8];
    R[2] = L[3] * L[7] - L[4] * L[6];
    R[3] = L[7] * L[2] - L[8] * L[1];
    R[4] = L[8] * L[0] - L[6] * L[2];
    R[5] = L[6] * L[1] - L[7] * L[0];
    double t = 1.0 / (L[0] * L[4] * L[8] + L[1] * L[5] * L[6] + L[2] * L[3] * L[7] - L[0] * L[5] * L[7] -
                      L[1] * L[3] * L[8] - L[2] * L[4] * L[6]);
    for (int k = 0; k < 9; k++) R[k] *= t;
}

/* triplet list gate: the union of the forward and derivative gates */
__device__ __forceinline__ bool tgate(const BParams &P, const WarpWS &ws, int s0, int jj, int kk) {
    float4 d1 = ws.d[jj], d2 = ws.d[kk];
    int sj = ws.sp[jj], sk = ws.sp[kk];
    int p01 = s0 * s0 + sj * sj, p02 = s0 * s0 + sk * sk, p12 = sj * sj + sk * sk;
    float dx = d1.x - d2.x, dy = d1.y - d2.y, dz = d1.z - d2.z;
    float r3s = dx * dx + dy * dy + dz * dz;
    bool fwd = d1.w < P.f_rc2[p01] && d1.w < P.f_rc4[p01] && d2.w < P.f_rc4[p02] && r3s < P.f_rc4sq[p12];
    bool rev = d1.w < P.d_rc4 && d2.w < P.d_rc4 && r3s < P.d_rc4sq;
    return fwd || rev;
}

/* ---------------- one atom: descriptors, MLP, reverse pass (FP32) ---------------- */

template <int W>
__device__ void atom_pass(const BArgs &A, BShared<W> &sh, WarpWS &ws, int i, const float4 *nbd, const int *nbj,
                          double *virw) {
    const BParams &P = *A.P;
    const int lane = threadIdx.x & 31;
    const int n = sh.nn[i], s0 = sh.spc[i], ns = P.nspc, D = P.D, ng2 = P.ng2;
    if (lane == 0) {
        ws.work[0] += 1ull;
        ws.work[1] += (unsigned long long)n;
    }
    int ntrip = 0; /* forward triplets this lane evaluated */
    /* stage neighbours stably sorted by relative species: counts and ranks
     * from warp ballots, one round per 32 neighbours */
    int cnt[4] = {0, 0, 0, 0};
    for (int base = 0; base < n; base += 32) {
        const int t = base + lane;
        const int ds = t < n ? (sh.spc[nbj[i * BMAXNB + t]] - s0 + ns) % ns : -1;
#pragma unroll
        for (int v = 0; v < 4; v++) cnt[v] += __popc(__ballot_sync(FULLM, ds == v));
    }
    for (int t = lane; t < D; t += 32) ws.G[t] = 0.0f;
    if (lane < 4) {
        int o = 0;
        for (int v = 0; v < lane; v++) o += cnt[v];
        ws.seg[lane] = cnt[lane];
        ws.seg[4 + lane] = o;
    }
    __syncwarp();
    int run[4] = {0, 0, 0, 0};
    const unsigned below = (1u << lane) - 1u;
    for (int base = 0; base < n; base += 32) {
        const int t = base + lane;
        const int sp = t < n ? sh.spc[nbj[i * BMAXNB + t]] : 0;
        const int ds = t < n ? (sp - s0 + ns) % ns : -1;
        int dst = 0;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const unsigned m = __ballot_sync(FULLM, ds == v);
            if (ds == v) dst = ws.seg[4 + v] + run[v] + __popc(m & below);
            run[v] += __popc(m);
        }
        if (t < n) {
            const float4 dv = nbd[i * BMAXNB + t];
            ws.d[dst] = dv;
            ws.ir[dst] = 1.0f / dv.w;
            ws.j[dst] = nbj[i * BMAXNB + t];
            ws.sp[dst] = sp;
        }
    }
    __syncwarp();

    /* forward pairs: G2 sums per relative species v and function f in lane
     * accumulators (cell 16 v + f; cells 48-63 stay zero), then warp sums */
    float g2acc[64];
#pragma unroll
    for (int k = 0; k < 64; k++) g2acc[k] = 0.0f;
    double eu = 0.0;
    for (int t = lane; t < n; t += 32) {
        float4 dv = ws.d[t];
        float r = dv.w;
        int sj = ws.sp[t], p = s0 * s0 + sj * sj, ds1 = (sj - s0 + ns) % ns;
        float fa = fcutf(P.f_rc2[p], r);
        ws.fa[t] = fa;
        ws.fb[t] = fcutf(P.f_rc4[p], r);
#pragma unroll
        for (int e = 0; e < 8; e++) ws.P[t * 8 + e] = e < P.ne ? expf(-P.f_eta4[p][e] * r * r) : 0.0f;
        if (r < P.f_rc2[p]) {
#pragma unroll
            for (int f = 0; f < 16; f++) {
                if (f < ng2) {
                    float x = r - P.f_rs[p][f];
                    float val = fa * expf(-P.f_eta2[p][f] * (x * x));
#pragma unroll
                    for (int v = 0; v < 3; v++)
                        if (v == ds1) g2acc[16 * v + f] += val;
                }
            }
        }
        if (A.urep > 0.0) {
            double R = P.rm[s0] + P.rm[sj], rd = (double)r;
            if (rd < R) eu += A.urep * 0.5 * (1.0 + cospi(rd / R)) * R / rd;
        }
    }
    /* summed across the warp by recursive halving: lane l ends with cells
     * 2l and 2l+1 */
    warp_reduce64f(g2acc, lane);
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int cell = 2 * lane + h, v = cell >> 4, f = cell & 15;
        if (v < ns && f < ng2) ws.G[P.ind2[v] + f] = g2acc[h];
    }
    eu = bsum(eu);
    if (lane == 0) sh.eu[i] = eu;
    __syncwarp();

    /* triplets: per species block, list of accepted (j,k), FP32 terms, lane accumulators */
    int tl_pos = 0, whole = 1, blkid = 0;
    for (int a = 0; a < ns; a++)
        for (int b = a; b < ns; b++, blkid++) {
            float acc[BCELLS];
#pragma unroll
            for (int k = 0; k < BCELLS; k++) acc[k] = 0.0f;
            const int na = ws.seg[a], nb = ws.seg[b], oa = ws.seg[4 + a], ob = ws.seg[4 + b];
            int start = tl_pos;
            /* j and k species are fixed within the block: hoist their parameters */
            const int sja = (a + s0) % ns, skb = (b + s0) % ns;
            const int p01 = s0 * s0 + sja * sja, p02 = s0 * s0 + skb * skb, p12 = sja * sja + skb * skb;
            const float rc2_01 = P.f_rc2[p01], rc4_01 = P.f_rc4[p01], rc4_02 = P.f_rc4[p02];
            const float rc4sq_12 = P.f_rc4sq[p12], rc4_12 = P.f_rc4[p12];
            const float drc4 = P.d_rc4, drc4sq = P.d_rc4sq;
            float eta12[BNE];
#pragma unroll
            for (int e = 0; e < BNE; e++) eta12[e] = P.f_eta4[p12][e];
            /* candidates (row, col) of the block in row-major order, 32 per
             * round with every lane busy.  Mixed blocks: all na x nb, row =
             * (c + 0.5) / nb in FP32 is exact (the fraction stays >= 0.5 / nb
             * from an integer).  Same-species blocks: only col > row; row r
             * starts at r (2 na - r - 1) / 2, inverted with one square root
             * and corrected by one row either way (exact for na <= 96 under
             * +-2 ulp of sqrt error) */
            const bool tri = a == b;
            const int C = tri ? na * (na - 1) / 2 : na * nb;
            const float inv_nb = nb > 0 ? 1.0f / (float)nb : 0.0f, tb = (float)(2 * na - 1);
            int c = 0;
            for (;;) {
                int from = tl_pos;
                for (; c < C && tl_pos + 32 <= BTL; c += 32) {
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
                        const float4 d1 = ws.d[jj], d2 = ws.d[kk];
                        const float dx = d1.x - d2.x, dy = d1.y - d2.y, dz = d1.z - d2.z;
                        const float r3s = dx * dx + dy * dy + dz * dz;
                        ok = (d1.w < rc2_01 && d1.w < rc4_01 && d2.w < rc4_02 && r3s < rc4sq_12) ||
                             (d1.w < drc4 && d2.w < drc4 && r3s < drc4sq);
                    }
                    const unsigned m = __ballot_sync(FULLM, ok);
                    if (ok) ws.tl[tl_pos + __popc(m & ((1u << lane) - 1u))] = (unsigned)jj | ((unsigned)kk << 16);
                    tl_pos += __popc(m);
                }
                __syncwarp();
                for (int t = from + lane; t < tl_pos; t += 32) {
                    unsigned pk = ws.tl[t];
                    int jj = pk & 0xffff, kk = pk >> 16;
                    float4 d1 = ws.d[jj], d2 = ws.d[kk];
                    float dx = d1.x - d2.x, dy = d1.y - d2.y, dz = d1.z - d2.z;
                    float r3s = dx * dx + dy * dy + dz * dz, r3 = sqrtf(r3s);
                    if (!(d1.w < rc2_01 && d1.w < rc4_01 && d2.w < rc4_02 && r3s < rc4sq_12)) continue;
                    ntrip++;
                    float c = (d1.x * d2.x + d1.y * d2.y + d1.z * d2.z) * (ws.ir[jj] * ws.ir[kk]);
                    float A3 = 2.0f * ws.fa[jj] * ws.fb[kk] * fcutf(rc4_12, r3);
                    float lz[BNZL];
                    angularf(P, c, lz, nullptr);
                    const float4 *pj = reinterpret_cast<const float4 *>(ws.P + jj * 8);
                    const float4 *pk4 = reinterpret_cast<const float4 *>(ws.P + kk * 8);
                    const float4 ja = pj[0], jb = pj[1], ka = pk4[0], kb4 = pk4[1];
                    const float pjk[8] = {ja.x * ka.x, ja.y * ka.y, ja.z * ka.z, ja.w * ka.w,
                                          jb.x * kb4.x, jb.y * kb4.y, jb.z * kb4.z, jb.w * kb4.w};
#pragma unroll
                    for (int e = 0; e < BNE; e++) {
                        const float ex = A3 * pjk[e] * expf(-eta12[e] * r3s);
                        const float2 ex2 = make_float2(ex, ex);
                        /* paired FP32 FMAs: two grid cells per instruction */
#pragma unroll
                        for (int zl = 0; zl < BNZL; zl += 2) {
                            const float2 r = __ffma2_rn(ex2, make_float2(lz[zl], lz[zl + 1]),
                                                        make_float2(acc[e * BNZL + zl], acc[e * BNZL + zl + 1]));
                            acc[e * BNZL + zl] = r.x;
                            acc[e * BNZL + zl + 1] = r.y;
                        }
                    }
                }
                __syncwarp();
                if (c >= C) break;
                whole = 0;
                start = tl_pos = 0;
            }
            ws.blk[blkid][0] = start;
            ws.blk[blkid][1] = tl_pos;
            /* lane sums across the warp */
            warp_reduce64f(acc, lane);
            ws.red[2 * lane] = acc[0];
            ws.red[2 * lane + 1] = acc[1];
            __syncwarp();
            {
                const int base = P.ind4[a * a + b * b];
                for (int f = lane; f < P.ng4; f += 32) ws.G[base + f] += ws.red[P.g4_cell[f]];
            }
            __syncwarp();
        }

    /* MLP forward and dE/dG (src/nmlp.c:367-431) */
    const int h1 = P.h1, h2 = P.h2;
    const float *net = A.W + P.w_off[s0];
    const float *off = net, *W0 = off + D, *b0 = W0 + h1 * D, *W1 = b0 + h1, *b1 = W1 + h2 * h1, *W2 = b1 + h2,
                *b2 = W2 + h2;
    float *H1 = ws.h, *Dl1 = ws.h + 2 * MB_MAXH;
    if (h1 <= 16) {
        /* every hidden unit's partial sum in each lane, then one reduction */
        float acc[16];
#pragma unroll
        for (int m = 0; m < 16; m++) acc[m] = 0.0f;
        for (int l = lane; l < D; l += 32) {
            const float x = ws.G[l] - off[l];
#pragma unroll
            for (int m = 0; m < 16; m++)
                if (m < h1) acc[m] += x * W0[m * D + l];
        }
        const float tot = warp_reduce16f(acc, lane);
        const int cell = (lane >> 1) & 15;
        if (!(lane & 1) && cell < h1) H1[cell] = tanhf(b0[cell] + tot);
    } else {
        for (int m = 0; m < h1; m++) {
            float acc = 0.0f;
            for (int l = lane; l < D; l += 32) acc += (ws.G[l] - off[l]) * W0[m * D + l];
            acc = bsumf(acc);
            if (lane == 0) H1[m] = tanhf(b0[m] + acc);
        }
    }
    __syncwarp();
    float v = 0.0f;
    if (lane < h2) {
        v = b1[lane];
        for (int k = 0; k < h1; k++) v += H1[k] * W1[lane * h1 + k];
        v = tanhf(v);
    }
    float e = lane < h2 ? v * W2[lane] : 0.0f;
    e = bsumf(e);
    if (lane == 0) sh.ea[i] = (double)b2[0] + (double)e;
    float dl2 = lane < h2 ? W2[lane] * (1.0f - v * v) : 0.0f;
    float dl1 = 0.0f;
    for (int m = 0; m < h2; m++) {
        float t = __shfl_sync(FULLM, dl2, m);
        if (lane < h1) dl1 += t * W1[m * h1 + lane];
    }
    if (lane < h1) Dl1[lane] = dl1 * (1.0f - H1[lane] * H1[lane]);
    __syncwarp();
    for (int l = lane; l < D; l += 32) {
        float g = 0.0f;
        for (int k = 0; k < h1; k++) g += Dl1[k] * W0[k * D + l];
        ws.G[l] = g;
    }
    __syncwarp();

    /* reverse pairs (species-0 derivative parameters) */
    float fi0 = 0.0f, fi1 = 0.0f, fi2 = 0.0f;
    /* the repulsion's force on atom i, kept in FP64 to the structure's
     * force array: at short distances it is the largest term (hundreds of
     * eV/A) and an FP32 sum of it would carry most of the rounding */
    double fu0 = 0.0, fu1 = 0.0, fu2 = 0.0;
    double vr[6] = {0, 0, 0, 0, 0, 0};
    for (int t = lane; t < n; t += 32) {
        float4 d = ws.d[t];
        float r = d.w, ir = ws.ir[t];
        float f4, df4, f2, df2;
        fcutf_d(P.d_rc4, r, f4, df4);
        fcutf_d(P.d_rc2, r, f2, df2);
        ws.fa[t] = f4;
        ws.fb[t] = df4;
#pragma unroll
        for (int q = 0; q < 8; q++) ws.P[t * 8 + q] = q < P.ne ? expf(-P.d_eta4[q] * r * r) : 0.0f;
        int ds1 = (ws.sp[t] - s0 + ns) % ns;
        const float *gg = ws.G + P.ind2[ds1];
        float cp = 0.0f;
        for (int f = 0; f < ng2; f++) {
            float x = r - P.d_rs[f], eta = P.d_eta2[f];
            cp += gg[f] * expf(-eta * x * x) * (-2.0f * eta * x * f2 + df2);
        }
        float cr = cp * ir;
        float v0 = cr * d.x, v1 = cr * d.y, v2 = cr * d.z;
        fi0 += v0; fi1 += v1; fi2 += v2;
        ws.Fnb[3 * t] = -v0; ws.Fnb[3 * t + 1] = -v1; ws.Fnb[3 * t + 2] = -v2;
        if (A.urep > 0.0) {
            double R = P.rm[s0] + P.rm[ws.sp[t]], rd = (double)r;
            if (rd < R) {
                double sn, cs;
                sincospi(rd / R, &sn, &cs);
                double fu = 0.5 * (1.0 + cs), dfu = -0.5 * CUDART_PI / R * sn;
                double tu = -2.0 * A.urep * R / (rd * rd) * (-fu / rd + dfu);
                fu0 -= tu * d.x; fu1 -= tu * d.y; fu2 -= tu * d.z;
                vr[0] += 0.5 * tu * d.x * d.x; vr[1] += 0.5 * tu * d.y * d.y; vr[2] += 0.5 * tu * d.z * d.z;
                vr[3] += 0.5 * tu * d.x * d.y; vr[4] += 0.5 * tu * d.y * d.z; vr[5] += 0.5 * tu * d.z * d.x;
            }
        }
    }
    __syncwarp();
    {
        const int t = __reduce_add_sync(FULLM, (unsigned)ntrip);
        if (lane == 0) ws.work[2] += (unsigned long long)t;
    }

    /* reverse triplets, reusing the lists when they fit */
    blkid = 0;
    const float drc4 = P.d_rc4, drc4sq = P.d_rc4sq;
    float deta[BNE];
#pragma unroll
    for (int q = 0; q < BNE; q++) deta[q] = P.d_eta4[q];
    for (int a = 0; a < ns; a++)
        for (int b = a; b < ns; b++, blkid++) {
            const int base = P.ind4[a * a + b * b];
            for (int t = lane; t < BCELLS; t += 32) ws.grid[t] = 0.0f;
            __syncwarp();
            for (int f = lane; f < P.ng4; f += 32) atomicAdd(&ws.grid[P.g4_cell[f]], ws.G[base + f]);
            __syncwarp();
            const int na = ws.seg[a], nb = ws.seg[b], oa = ws.seg[4 + a], ob = ws.seg[4 + b];
            int row = 0, lo = whole ? ws.blk[blkid][0] : 0, hi = whole ? ws.blk[blkid][1] : 0;
            for (;;) {
                if (!whole) {
                    hi = 0;
                    for (; row < na; row++) {
                        int jj = oa + row, k0 = (a == b) ? row + 1 : 0;
                        if (hi + (nb - k0) > BTL) break;
                        for (int kb = k0; kb < nb; kb += 32) {
                            int kk = ob + kb + lane;
                            bool ok = false;
                            if (kb + lane < nb) ok = tgate(P, ws, s0, jj, kk);
                            unsigned m = __ballot_sync(FULLM, ok);
                            if (ok) ws.tl[hi + __popc(m & ((1u << lane) - 1u))] = (unsigned)jj | ((unsigned)kk << 16);
                            hi += __popc(m);
                        }
                    }
                    lo = 0;
                    __syncwarp();
                }
                {
                    /* 32 consecutive list entries per round: the list runs row by
                     * row, so within a round the lanes of one row j are contiguous
                     * and their k differ (the k-side atomics rarely collide); the
                     * j-side forces are summed per row by a segmented warp sum and
                     * added by the row's first lane */
                    for (int base = lo; base < hi; base += 32) {
                        const int t = base + lane;
                        int jj = -1 - lane, kk = 0;
                        float g1x = 0.0f, g1y = 0.0f, g1z = 0.0f;
                        if (t < hi) {
                            const unsigned pk = ws.tl[t];
                            jj = pk & 0xffff;
                            kk = pk >> 16;
                        }
                        const float4 d1 = ws.d[max(jj, 0)], d2 = ws.d[kk];
                        const float wx = d2.x - d1.x, wy = d2.y - d1.y, wz = d2.z - d1.z;
                        const float r3s = wx * wx + wy * wy + wz * wz, r3 = sqrtf(r3s);
                        if (t < hi && d1.w < drc4 && d2.w < drc4 && r3s < drc4sq) {
                            float r1 = d1.w, r2 = d2.w, ir1 = ws.ir[jj], ir2 = ws.ir[kk], ir3 = 1.0f / r3;
                            float c = (d1.x * d2.x + d1.y * d2.y + d1.z * d2.z) * (ir1 * ir2);
                            float f3, df3;
                            fcutf_d(drc4, r3, f3, df3);
                            float f1 = ws.fa[jj], df1 = ws.fb[jj], f2 = ws.fa[kk], df2 = ws.fb[kk];
                            float lz[BNZL], lzp[BNZL];
                            angularf(P, c, lz, lzp);
                            float Q = 0.0f, Qe = 0.0f, Qc = 0.0f;
                            const float4 *pj = reinterpret_cast<const float4 *>(ws.P + jj * 8);
                            const float4 *pk4 = reinterpret_cast<const float4 *>(ws.P + kk * 8);
                            const float4 ja = pj[0], jb = pj[1], ka = pk4[0], kb4 = pk4[1];
                            const float pjk[8] = {ja.x * ka.x, ja.y * ka.y, ja.z * ka.z, ja.w * ka.w,
                                                  jb.x * kb4.x, jb.y * kb4.y, jb.z * kb4.z, jb.w * kb4.w};
                            const float4 *g4 = reinterpret_cast<const float4 *>(ws.grid);
#pragma unroll
                            for (int q = 0; q < BNE; q++) {
                                const float ex = pjk[q] * expf(-deta[q] * r3s);
                                const float4 ga = g4[2 * q], gb = g4[2 * q + 1];
                                const float cg[8] = {ga.x, ga.y, ga.z, ga.w, gb.x, gb.y, gb.z, gb.w};
                                /* (u, v) = sum over cells of cg * (lz, lz') with paired FMAs */
                                float2 uv = make_float2(0.0f, 0.0f);
#pragma unroll
                                for (int zl = 0; zl < BNZL; zl++)
                                    uv = __ffma2_rn(make_float2(cg[zl], cg[zl]), make_float2(lz[zl], lzp[zl]), uv);
                                const float u = uv.x, vv = uv.y;
                                Q += ex * u;
                                Qe += deta[q] * ex * u;
                                Qc += ex * vv;
                            }
                            float Af = 2.0f * f1 * f2 * f3;
                            float T1 = 2.0f * df1 * f2 * f3 * Q - 2.0f * r1 * Af * Qe;
                            float T2 = 2.0f * f1 * df2 * f3 * Q - 2.0f * r2 * Af * Qe;
                            float T3 = 2.0f * f1 * f2 * df3 * Q - 2.0f * r3 * Af * Qe;
                            float Tc = Af * Qc;
                            float a11 = T1 * ir1 - Tc * c * ir1 * ir1, a22 = T2 * ir2 - Tc * c * ir2 * ir2;
                            float a12 = Tc * ir1 * ir2, a3 = T3 * ir3;
                            g1x = a11 * d1.x + a12 * d2.x - a3 * wx;
                            g1y = a11 * d1.y + a12 * d2.y - a3 * wy;
                            g1z = a11 * d1.z + a12 * d2.z - a3 * wz;
                            const float g2x = a22 * d2.x + a12 * d1.x + a3 * wx;
                            const float g2y = a22 * d2.y + a12 * d1.y + a3 * wy;
                            const float g2z = a22 * d2.z + a12 * d1.z + a3 * wz;
                            fi0 += g1x + g2x; fi1 += g1y + g2y; fi2 += g1z + g2z;
                            atomicAdd(&ws.Fnb[3 * kk], -g2x);
                            atomicAdd(&ws.Fnb[3 * kk + 1], -g2y);
                            atomicAdd(&ws.Fnb[3 * kk + 2], -g2z);
                        }
#pragma unroll
                        for (int o = 1; o < 32; o <<= 1) {
                            const float x = __shfl_down_sync(FULLM, g1x, o), y = __shfl_down_sync(FULLM, g1y, o),
                                        z = __shfl_down_sync(FULLM, g1z, o);
                            const int jn = __shfl_down_sync(FULLM, jj, o);
                            if (lane + o < 32 && jn == jj) {
                                g1x += x;
                                g1y += y;
                                g1z += z;
                            }
                        }
                        const int jp = __shfl_up_sync(FULLM, jj, 1);
                        if (jj >= 0 && (lane == 0 || jp != jj)) {
                            atomicAdd(&ws.Fnb[3 * jj], -g1x);
                            atomicAdd(&ws.Fnb[3 * jj + 1], -g1y);
                            atomicAdd(&ws.Fnb[3 * jj + 2], -g1z);
                        }
                    }
                }
                __syncwarp();
                if (whole || row >= na) break;
            }
        }
    /* virial of atom i's energy: every neighbour force Fnb[t] (pairs and
     * triplets) times its displacement, summed in FP64 -- the same sum as
     * -(dE/dd) (x) d taken term by term, formed once per neighbour */
    for (int t = lane; t < n; t += 32) {
        const float4 d = ws.d[t];
        const double fx = ws.Fnb[3 * t], fy = ws.Fnb[3 * t + 1], fz = ws.Fnb[3 * t + 2];
        vr[0] += fx * d.x; vr[1] += fy * d.y; vr[2] += fz * d.z;
        vr[3] += fx * d.y; vr[4] += fy * d.z; vr[5] += fz * d.x;
    }
    /* gather: atom i and its neighbours into the structure's force array */
    {
        const double s0x = bsum((double)fi0 + fu0), s0y = bsum((double)fi1 + fu1), s0z = bsum((double)fi2 + fu2);
        if (lane == 0) {
            atomicAdd(&sh.F[3 * i], s0x);
            atomicAdd(&sh.F[3 * i + 1], s0y);
            atomicAdd(&sh.F[3 * i + 2], s0z);
        }
    }
    for (int t = lane; t < n; t += 32) {
        int j = ws.j[t];
        atomicAdd(&sh.F[3 * j], (double)ws.Fnb[3 * t]);
        atomicAdd(&sh.F[3 * j + 1], (double)ws.Fnb[3 * t + 1]);
        atomicAdd(&sh.F[3 * j + 2], (double)ws.Fnb[3 * t + 2]);
    }
#pragma unroll
    for (int k = 0; k < 6; k++) virw[k] += bsum(vr[k]);
    __syncwarp();
}

/* ---------------- one evaluation of the structure at DOF vector dof ---------------- */

/* One CTA's share of an evaluation: every atom's position from the DOF
 * vector, then neighbour lists and the per-atom pass for atoms
 * rank W + w (mod C W), i.e. warp w of cluster rank `rank`.  Leaves
 * partial forces in sh.F (all atoms), ea/eu of its own atoms, the per-warp
 * virials in sh.vir and any overflow in sh.flag. */
template <int W, int C>
__device__ void eval_part(const BArgs &A, BShared<W> &sh, const double *dof, int rank) {
    const BParams &P = *A.P;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, N = sh.N, rlxt = A.rlxt;
    const int first_atom = rank * W + w, stride = C * W;
    float4 *nbd = A.nbd + (size_t)blockIdx.x * BMAXN * BMAXNB;
    int *nbj = A.nbj + (size_t)blockIdx.x * BMAXN * BMAXNB;
    /* structure from the DOF vector (BUF_STR, src/cmin.c:54-88) */
    if (tid == 0) {
        if (rlxt != 2) {
            const double *q = dof + 3 * N;
            sh.L[0] = q[0]; sh.L[4] = q[1]; sh.L[8] = q[2]; sh.L[1] = q[3]; sh.L[5] = q[4];
            sh.L[6] = q[5]; sh.L[3] = q[6]; sh.L[7] = q[7]; sh.L[2] = q[8];
        }
        reciprocal9(sh.L, sh.R);
    }
    __syncthreads();
    for (int a = tid; a < N; a += blockDim.x) {
        double f[3];
        for (int q = 0; q < 3; q++) f[q] = dof[3 * a + q] - floor(dof[3 * a + q]);
        for (int q = 0; q < 3; q++) sh.xc[3 * a + q] = f[0] * sh.L[q] + f[1] * sh.L[3 + q] + f[2] * sh.L[6 + q];
        sh.F[3 * a] = sh.F[3 * a + 1] = sh.F[3 * a + 2] = 0.0;
    }
    if (tid < 6) sh.uvir[tid] = 0.0;
    __syncthreads();
    /* neighbour lists: every (atom, image) within Rc, displacement in FP64 */
    int nq[3];
    for (int q = 0; q < 3; q++) {
        double len = sqrt(sh.R[3 * q] * sh.R[3 * q] + sh.R[3 * q + 1] * sh.R[3 * q + 1] + sh.R[3 * q + 2] * sh.R[3 * q + 2]);
        nq[q] = (int)ceil(P.rc * len);
    }
    const int w0 = 2 * nq[0] + 1, w1 = 2 * nq[1] + 1, w2 = 2 * nq[2] + 1, nimg = w0 * w1 * w2;
    const double rc2 = P.rc * P.rc;
    if (nimg <= 32 * BIMG) {
        /* each lane holds the Cartesian shifts of images lane, lane+32, ...;
         * candidates in the order (j, image), as the general loop below */
        double shx[BIMG], shy[BIMG], shz[BIMG];
        unsigned zero = 0; /* bit t: image lane + 32 t is the unshifted cell */
#pragma unroll
        for (int t = 0; t < BIMG; t++) {
            const int im = lane + 32 * t;
            const int c2 = im % w2 - nq[2], u = im / w2, c1 = u % w1 - nq[1], c0 = u / w1 - nq[0];
            shx[t] = c0 * sh.L[0] + c1 * sh.L[3] + c2 * sh.L[6];
            shy[t] = c0 * sh.L[1] + c1 * sh.L[4] + c2 * sh.L[7];
            shz[t] = c0 * sh.L[2] + c1 * sh.L[5] + c2 * sh.L[8];
            if (c0 == 0 && c1 == 0 && c2 == 0) zero |= 1u << t;
        }
        for (int i = first_atom; i < N; i += stride) {
            int count = 0;
            const double xi0 = sh.xc[3 * i], xi1 = sh.xc[3 * i + 1], xi2 = sh.xc[3 * i + 2];
            for (int j = 0; j < N; j++) {
                const double b0 = sh.xc[3 * j] - xi0, b1 = sh.xc[3 * j + 1] - xi1, b2 = sh.xc[3 * j + 2] - xi2;
#pragma unroll
                for (int t = 0; t < BIMG; t++) {
                    if (32 * t >= nimg) break;
                    const int im = lane + 32 * t;
                    const double d0 = b0 + shx[t], d1 = b1 + shy[t], d2 = b2 + shz[t];
                    const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
                    const bool ok = im < nimg && r2 < rc2 && !(j == i && ((zero >> t) & 1u));
                    const unsigned m = __ballot_sync(FULLM, ok);
                    const int pos = count + __popc(m & ((1u << lane) - 1u));
                    if (ok && pos < BMAXNB) {
                        nbj[i * BMAXNB + pos] = j;
                        nbd[i * BMAXNB + pos] = make_float4((float)d0, (float)d1, (float)d2, (float)sqrt(r2));
                    }
                    count += __popc(m);
                }
            }
            if (lane == 0) {
                sh.nn[i] = count < BMAXNB ? count : BMAXNB;
                if (count > BMAXNB) sh.flag = 2;
            }
        }
    } else
    for (int i = first_atom; i < N; i += stride) {
        int count = 0;
        const double xi0 = sh.xc[3 * i], xi1 = sh.xc[3 * i + 1], xi2 = sh.xc[3 * i + 2];
        for (int base = 0; base < N * nimg; base += 32) {
            int cidx = base + lane;
            bool ok = false;
            double d0 = 0, d1 = 0, d2 = 0, r2 = 0;
            int j = 0;
            if (cidx < N * nimg) {
                j = cidx / nimg;
                int im = cidx % nimg, c2 = im % w2 - nq[2], t = im / w2, c1 = t % w1 - nq[1], c0 = t / w1 - nq[0];
                if (!(j == i && c0 == 0 && c1 == 0 && c2 == 0)) {
                    d0 = c0 * sh.L[0] + c1 * sh.L[3] + c2 * sh.L[6] + sh.xc[3 * j] - xi0;
                    d1 = c0 * sh.L[1] + c1 * sh.L[4] + c2 * sh.L[7] + sh.xc[3 * j + 1] - xi1;
                    d2 = c0 * sh.L[2] + c1 * sh.L[5] + c2 * sh.L[8] + sh.xc[3 * j + 2] - xi2;
                    r2 = d0 * d0 + d1 * d1 + d2 * d2;
                    ok = r2 < rc2;
                }
            }
            unsigned m = __ballot_sync(FULLM, ok);
            int pos = count + __popc(m & ((1u << lane) - 1u));
            if (ok && pos < BMAXNB) {
                nbj[i * BMAXNB + pos] = j;
                nbd[i * BMAXNB + pos] = make_float4((float)d0, (float)d1, (float)d2, (float)sqrt(r2));
            }
            count += __popc(m);
        }
        if (lane == 0) {
            sh.nn[i] = count < BMAXNB ? count : BMAXNB;
            if (count > BMAXNB) sh.flag = 2;
        }
    }
    __syncthreads();
    /* descriptors, MLP and forces, one warp per atom */
    double virw[6] = {0, 0, 0, 0, 0, 0};
    for (int i = first_atom; i < N; i += stride) atom_pass(A, sh, sh.ws[w], i, nbd, nbj, virw);
    if (lane == 0)
        for (int k = 0; k < 6; k++) sh.vir[w][k] = virw[k];
    __syncthreads();
}

/* Rank 0 of a cluster, after the other ranks' parts are complete: their
 * partial forces and virials added to its own in rank order, per-atom
 * energies taken from each atom's owner, overflow flags joined. */
template <int W, int C>
__device__ void eval_combine(BShared<W> &sh) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int tid = threadIdx.x, N = sh.N;
    for (int a = tid; a < N; a += blockDim.x) {
        const int owner = (a % (C * W)) / W;
        if (owner != 0) {
            const BShared<W> *ro = cl.map_shared_rank(&sh, owner);
            sh.ea[a] = ro->ea[a];
            sh.eu[a] = ro->eu[a];
        }
        for (int q = 0; q < 3; q++) {
            double f = sh.F[3 * a + q];
            for (int r = 1; r < C; r++) f += cl.map_shared_rank(&sh, r)->F[3 * a + q];
            sh.F[3 * a + q] = f;
        }
    }
    for (int k = tid; k < 6 * W; k += blockDim.x) {
        double v = sh.vir[k / 6][k % 6];
        for (int r = 1; r < C; r++) v += cl.map_shared_rank(&sh, r)->vir[k / 6][k % 6];
        sh.vir[k / 6][k % 6] = v;
    }
    if (tid == 0)
        for (int r = 1; r < C; r++) sh.flag |= cl.map_shared_rank(&sh, r)->flag;
    __syncthreads();
}

/* FP64 reductions of a complete evaluation (rank 0). */
template <int W>
__device__ double eval_finish(const BArgs &A, BShared<W> &sh, double *gout) {
    const int tid = threadIdx.x, N = sh.N, rlxt = A.rlxt;
    /* FP64 reductions, enthalpy and the DOF gradient (cdfunc_gsl, src/cmin.c:107-166) */
    if (tid == 0) {
        double E = 0.0, U[6];
        double mag = 0.0;
        for (int a = 0; a < N; a++) {
            E += sh.ea[a] + sh.eu[a];
            mag += fabs(sh.ea[a]);
        }
        /* rounding floor of the enthalpy: the per-atom energies come from FP32
         * descriptors and MLP, a few ulps each */
        sh.scal[3] = 4.0 * 1.1920929e-7 * mag;
        for (int k = 0; k < 6; k++) {
            U[k] = 0.0;
            for (int ww = 0; ww < W; ww++) U[k] += sh.vir[ww][k];
        }
        const double *L = sh.L;
        double V = fabs(L[0] * L[4] * L[8] + L[2] * L[3] * L[7] + L[1] * L[5] * L[6] - L[0] * L[5] * L[7] -
                        L[1] * L[3] * L[8] - L[2] * L[4] * L[6]);
        double pv = A.p_ev * V;
        sh.scal[0] = E + pv;
        sh.scal[4] = pv;
        for (int q = 0; q < 3; q++) U[q] -= pv;
        for (int k = 0; k < 6; k++) sh.uvir[k] = U[k];
        double mu = 0.0;
        if (rlxt != 2)
            for (int k = 0; k < 6; k++) mu = fmax(mu, fabs(U[k]) / N);
        sh.scal[2] = mu;
    }
    __syncthreads();
    double mf = 0.0;
    for (int a = tid; a < N; a += blockDim.x)
        for (int q = 0; q < 3; q++) {
            double gq = 0.0;
            for (int k = 0; k < 3; k++) gq -= sh.F[3 * a + k] * sh.L[3 * q + k];
            gout[3 * a + q] = fabs(gq) < 1e-10 ? 0.0 : gq;
            mf = fmax(mf, fabs(sh.F[3 * a + q]));
        }
    mf = cta_max(sh, mf);
    if (tid == 0) {
        sh.scal[1] = mf;
        if (rlxt != 2) {
            const double *U = sh.uvir, *R = sh.R;
            double *q = gout + 3 * N;
            q[0] = -(U[0] * R[0] + U[3] * R[1] + U[5] * R[2]);
            q[1] = -(U[3] * R[3] + U[1] * R[4] + U[4] * R[5]);
            q[2] = -(U[5] * R[6] + U[4] * R[7] + U[2] * R[8]);
            q[3] = -(U[3] * R[0] + U[1] * R[1] + U[4] * R[2]);
            q[4] = -(U[5] * R[3] + U[4] * R[4] + U[2] * R[5]);
            q[5] = -(U[0] * R[6] + U[3] * R[7] + U[5] * R[8]);
            q[6] = -(U[0] * R[3] + U[3] * R[4] + U[5] * R[5]);
            q[7] = -(U[3] * R[6] + U[1] * R[7] + U[4] * R[8]);
            q[8] = -(U[5] * R[0] + U[4] * R[1] + U[2] * R[2]);
            for (int k = 0; k < 9; k++)
                if (fabs(q[k]) < 1e-10) q[k] = 0.0;
        }
        atomicAdd((unsigned long long *)A.evals, 1ull);
    }
    __syncthreads();
    return sh.scal[0];
}

/* Returns H; gradient into gout; sh.scal[1] = max|F|, sh.scal[2] = max|U-pV|/N.
 * Called by rank 0 only.  With C > 1 the evaluation is posted to the other
 * ranks (cluster barrier), every rank evaluates its atoms, and a second
 * barrier precedes the combination: two barriers per evaluation, matched
 * one for one by the other ranks' command loop. */
template <int W, int C>
__device__ double evaluate(const BArgs &A, BShared<W> &sh, const double *dof, double *gout) {
    if constexpr (C > 1) {
        if (threadIdx.x == 0) sh.cmd_dof = dof == sh.x ? 0 : 1;
        cooperative_groups::this_cluster().sync();
    }
    eval_part<W, C>(A, sh, dof, 0);
    if constexpr (C > 1) {
        cooperative_groups::this_cluster().sync();
        eval_combine<W, C>(sh);
    }
    return eval_finish<W>(A, sh, gout);
}

/* Ranks 1..C-1 of a cluster: wait for rank 0's command, copy its DOF
 * vector, evaluate their atoms, and meet rank 0 at the second barrier.
 * Rank 0 posts structure -1 when the queue is empty; one last barrier
 * keeps every rank's shared memory alive until all have read it. */
template <int W, int C>
__device__ void cluster_worker(const BArgs &A, BShared<W> &sh, int rank) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int tid = threadIdx.x;
    int cur = -1;
    for (;;) {
        cl.sync();
        const BShared<W> *r0 = cl.map_shared_rank(&sh, 0);
        const int s = r0->cmd_s, which = r0->cmd_dof;
        if (s < 0) break;
        const int N = A.nat[s], o = A.off[s];
        const int n = 3 * N + (A.rlxt == 3 ? 9 : 0);
        if (s != cur) {
            if (tid == 0) {
                sh.N = N;
                sh.ndof = n;
                sh.flag = 0;
                for (int k = 0; k < 9; k++) sh.L[k] = A.lat[9 * s + k];
            }
            for (int a = tid; a < N; a += blockDim.x) sh.spc[a] = A.spc[o + a];
            cur = s;
        }
        const double *src = which ? r0->xt : r0->x;
        for (int k = tid; k < n; k += blockDim.x) sh.x[k] = src[k];
        __syncthreads();
        eval_part<W, C>(A, sh, sh.x, rank);
        cl.sync();
    }
    cl.sync();
}

/* each warp's work counts into the launch's totals (once per warp, at exit) */
template <int W>
__device__ void flush_work(const BArgs &A, BShared<W> &sh) {
    if ((threadIdx.x & 31) == 0 && A.work) {
        const WarpWS &ws = sh.ws[threadIdx.x >> 5];
        for (int k = 0; k < 3; k++) atomicAdd(A.work + k, ws.work[k]);
    }
}

/* cubic (or quadratic without db) minimiser on [lo,hi] (Fletcher, sec. 2.6) */
__device__ double interp_min(double a, double fa, double da, double b, double fb, double db, double lo, double hi) {
    double w = b - a;
    if (w == 0.0) return a;
    double zlo = (lo - a) / w, zhi = (hi - a) / w;
    if (zlo > zhi) { double t = zlo; zlo = zhi; zhi = t; }
    double c0 = fa, c1 = da * w, c2 = 3.0 * (fb - fa) - 2.0 * c1 - db * w, c3 = c1 + db * w - 2.0 * (fb - fa);
    double cand[4];
    int nc = 0;
    cand[nc++] = zlo;
    cand[nc++] = zhi;
    if (c3 != 0.0) {
        double disc = 4.0 * c2 * c2 - 12.0 * c3 * c1;
        if (disc >= 0.0) {
            double sq = sqrt(disc), q = -0.5 * (2.0 * c2 + (c2 >= 0.0 ? sq : -sq));
            if (q != 0.0) {
                cand[nc++] = q / (3.0 * c3);
                cand[nc++] = c1 / q;
            }
        }
    } else if (c2 > 0.0) {
        cand[nc++] = -c1 / (2.0 * c2);
    }
    double best = zlo, fbest = 1e300;
    for (int k = 0; k < nc; k++) {
        double z = cand[k];
        if (!(z >= zlo && z <= zhi)) continue;
        double fz = c0 + z * (c1 + z * (c2 + z * c3));
        if (fz < fbest) { fbest = fz; best = z; }
    }
    return a + best * w;
}

__device__ void vcopy(double *dst, const double *src, int n) {
    for (int k = threadIdx.x; k < n; k += blockDim.x) dst[k] = src[k];
}

template <int W, int C>
__global__ void __launch_bounds__(W * 32) k_relax_batch(BArgs A) {
    extern __shared__ __align__(16) char smem_raw[];
    BShared<W> &sh = *reinterpret_cast<BShared<W> *>(smem_raw);
    const int tid = threadIdx.x;
    if ((tid & 31) == 0)
        for (int k = 0; k < 3; k++) sh.ws[tid >> 5].work[k] = 0ull;
    /* (every warp's first atom pass comes after a CTA or cluster barrier) */
    if constexpr (C > 1) {
        const int rank = (int)cooperative_groups::this_cluster().block_rank();
        if (rank != 0) {
            cluster_worker<W, C>(A, sh, rank);
            flush_work(A, sh);
            return;
        }
    }
    double *H = A.hmat + (size_t)blockIdx.x * BMAXDOF * BMAXDOF;
    const double rho = 0.01, tau1 = 9.0, tau2 = 0.05, tau3 = 0.5;
    for (;;) {
        if (tid == 0) sh.s = atomicAdd(A.queue, 1);
        __syncthreads();
        if (sh.s >= A.S) break;
        const int s = A.order[sh.s];
        const int N = A.nat[s], o = A.off[s], rlxt = A.rlxt;
        const int n = 3 * N + (rlxt == 3 ? 9 : 0);
        if (tid == 0) {
            sh.cmd_s = s;
            sh.N = N;
            sh.ndof = n;
            sh.flag = 0;
            for (int k = 0; k < 9; k++) sh.L[k] = A.lat[9 * s + k];
            reciprocal9(sh.L, sh.R);
        }
        __syncthreads();
        /* DOF vector: fractional coordinates then lattice (STR_BUF, src/cmin.c:22-52) */
        for (int a = tid; a < N; a += blockDim.x) {
            sh.spc[a] = A.spc[o + a];
            for (int q = 0; q < 3; q++) {
                const double *xa = A.x + 3 * (size_t)(o + a);
                sh.x[3 * a + q] = xa[0] * sh.R[3 * q] + xa[1] * sh.R[3 * q + 1] + xa[2] * sh.R[3 * q + 2];
            }
        }
        if (tid == 0 && rlxt == 3) {
            double *q = sh.x + 3 * N;
            q[0] = sh.L[0]; q[1] = sh.L[4]; q[2] = sh.L[8]; q[3] = sh.L[1]; q[4] = sh.L[5];
            q[5] = sh.L[6]; q[6] = sh.L[3]; q[7] = sh.L[7]; q[8] = sh.L[2];
        }
        for (int k = tid; k < n * n; k += blockDim.x) H[k] = (k / n == k % n) ? 1.0 : 0.0;
        __syncthreads();
        double f = evaluate<W, C>(A, sh, sh.x, sh.g), fprev = f;
        double maxf = sh.scal[1], maxu = sh.scal[2];
        int first = 1, iter = 0, status = 1;
        if (sh.flag) status = 2;
        else if (maxf < A.fmax && maxu < A.fmax) status = 0;
        while (status == 1 && iter < A.mitr) {
            iter++;
            /* p = -H g; H is exactly symmetric (see the update below), so row r
             * is read as column r: consecutive threads read consecutive
             * elements */
            for (int r = tid; r < n; r += blockDim.x) {
                double t = 0.0;
                for (int c = 0; c < n; c++) t += H[c * n + r] * sh.g[c];
                sh.p[r] = -t;
            }
            __syncthreads();
            double dphi0 = 0.0, pp = 0.0;
            for (int k = tid; k < n; k += blockDim.x) { dphi0 += sh.g[k] * sh.p[k]; }
            dphi0 = cta_sum(sh, dphi0);
            if (!(dphi0 < 0.0)) {
                for (int k = tid; k < n * n; k += blockDim.x) H[k] = (k / n == k % n) ? 1.0 : 0.0;
                for (int k = tid; k < n; k += blockDim.x) sh.p[k] = -sh.g[k];
                __syncthreads();
                first = 1;
                dphi0 = 0.0;
                for (int k = tid; k < n; k += blockDim.x) dphi0 += sh.g[k] * sh.p[k];
                dphi0 = cta_sum(sh, dphi0);
                if (!(dphi0 < 0.0)) { status = 0; break; } /* zero gradient: at a stationary point */
            }
            for (int k = tid; k < n; k += blockDim.x) pp += sh.p[k] * sh.p[k];
            pp = cta_sum(sh, pp);
            double alpha = first ? 0.01 / sqrt(pp) : 2.0 * (f - fprev) / dphi0;
            if (!first && (!(alpha > 0.0) || alpha > 1.0)) alpha = 1.0;
            /* Fletcher line search with energy and gradient at every trial */
            double ap = 0.0, fp = f, dp = dphi0, a = 0, fa = 0, da = 0, b = 0, fb = 0, db = 0;
            double a_maxf = maxf, a_maxu = maxu, ft = 0.0, dt;
            /* energy comparisons allow the FP32 rounding floor: below it only
             * the (accurate) directional derivative can tell progress */
            const double epsE = sh.scal[3];
            int phase = 0, done = 0, trial;
            vcopy(sh.xa, sh.x, n);
            vcopy(sh.ga, sh.g, n);
            __syncthreads();
            for (trial = 0; trial < 60 && !done; trial++) {
                for (int k = tid; k < n; k += blockDim.x) sh.xt[k] = sh.x[k] + alpha * sh.p[k];
                __syncthreads();
                ft = evaluate<W, C>(A, sh, sh.xt, sh.gt);
                double t = 0.0;
                for (int k = tid; k < n; k += blockDim.x) t += sh.gt[k] * sh.p[k];
                dt = cta_sum(sh, t);
                if (sh.flag) { done = 3; break; }
                const double mft = sh.scal[1], mut = sh.scal[2];
                int save_a = 0;
                double next = alpha;
                if (!isfinite(ft)) { done = 4; break; }
                if (phase == 0) {
                    if (ft > f + rho * alpha * dphi0 + epsE || (trial > 0 && ft >= fp + epsE)) {
                        a = ap; fa = fp; da = dp; b = alpha; fb = ft; db = dt;
                        phase = 1;
                    } else if (fabs(dt) <= -A.sigma * dphi0) {
                        done = 1;
                    } else if (dt >= 0.0) {
                        a = alpha; fa = ft; da = dt; b = ap; fb = fp; db = dp;
                        save_a = 1;
                        phase = 1;
                    } else {
                        next = interp_min(ap, fp, dp, alpha, ft, dt, 2.0 * alpha - ap, alpha + tau1 * (alpha - ap));
                        ap = alpha; fp = ft; dp = dt;
                        save_a = 1;
                    }
                } else {
                    if (ft > f + rho * alpha * dphi0 + epsE || ft >= fa + epsE) {
                        b = alpha; fb = ft; db = dt;
                    } else if (fabs(dt) <= -A.sigma * dphi0) {
                        done = 1;
                    } else {
                        if ((b - a) * dt >= 0.0) { b = a; fb = fa; db = da; }
                        a = alpha; fa = ft; da = dt;
                        save_a = 1;
                    }
                }
                if (save_a) {
                    vcopy(sh.xa, sh.xt, n);
                    vcopy(sh.ga, sh.gt, n);
                    a_maxf = mft;
                    a_maxu = mut;
                }
                if (done) {
                    maxf = mft;
                    maxu = mut;
                    break;
                }
                if (phase == 1) {
                    if (fabs((a - b) * da) <= 4.0 * 2.220446049250313e-16 * (fabs(f) + 1.0) || trial == 59) {
                        done = 2; /* interval exhausted: the best point stands */
                        break;
                    }
                    next = interp_min(a, fa, da, b, fb, db, a + tau2 * (b - a), b - tau3 * (b - a));
                }
                alpha = next;
                __syncthreads();
            }
            __syncthreads();
            if (done == 3) { status = 2; break; }
            if (done == 2 || done == 4 || done == 0) {
                /* accept the best bracketed point if it lowered the enthalpy */
                if (phase == 1 && a > 0.0 && fa < f + epsE) {
                    vcopy(sh.xt, sh.xa, n);
                    vcopy(sh.gt, sh.ga, n);
                    alpha = a;
                    ft = fa;
                    maxf = a_maxf;
                    maxu = a_maxu;
                    __syncthreads();
                } else if (!first) {
                    /* no acceptable step along the quasi-Newton direction:
                     * restart once from steepest descent before giving up */
                    for (int k = tid; k < n * n; k += blockDim.x) H[k] = (k / n == k % n) ? 1.0 : 0.0;
                    first = 1;
                    __syncthreads();
                    continue;
                } else {
                    status = 3;
                    break;
                }
            }
            /* BFGS update with s = alpha p, y = gt - g (Nocedal & Wright 6.17, 6.20) */
            for (int k = tid; k < n; k += blockDim.x) {
                sh.p[k] *= alpha;
                sh.hy[k] = sh.gt[k] - sh.g[k];
            }
            __syncthreads();
            double sy = 0.0, yy = 0.0;
            for (int k = tid; k < n; k += blockDim.x) { sy += sh.p[k] * sh.hy[k]; yy += sh.hy[k] * sh.hy[k]; }
            sy = cta_sum(sh, sy);
            yy = cta_sum(sh, yy);
            if (sy > 0.0) {
                if (first)
                    for (int k = tid; k < n * n; k += blockDim.x) H[k] = (k / n == k % n) ? sy / yy : 0.0;
                __syncthreads();
                /* Hy into g (g is replaced below) */
                for (int r = tid; r < n; r += blockDim.x) {
                    double t = 0.0;
                    for (int c = 0; c < n; c++) t += H[c * n + r] * sh.hy[c];
                    sh.g[r] = t;
                }
                __syncthreads();
                double yhy = 0.0;
                for (int k = tid; k < n; k += blockDim.x) yhy += sh.hy[k] * sh.g[k];
                yhy = cta_sum(sh, yhy);
                const double c1 = (sy + yhy) / (sy * sy);
                /* elements (r, c) and (c, r) get the same operations on the
                 * same values (products and the sum unfused, so no
                 * contraction rounds the two orders differently): H stays
                 * exactly symmetric */
                for (int k = tid; k < n * n; k += blockDim.x) {
                    int r = k / n, c = k % n;
                    const double pp = __dmul_rn(sh.p[r], sh.p[c]);
                    const double gp = __dadd_rn(__dmul_rn(sh.g[r], sh.p[c]), __dmul_rn(sh.p[r], sh.g[c]));
                    H[k] += c1 * pp - gp / sy;
                }
            }
            __syncthreads();
            vcopy(sh.x, sh.xt, n);
            vcopy(sh.g, sh.gt, n);
            __syncthreads();
            fprev = f;
            f = ft;
            first = 0;
            if (maxf < A.fmax && maxu < A.fmax) status = 0;
        }
        /* forces and virial of the final state, on request: the last
         * evaluation was at the final DOF vector only if no step was taken */
        if (A.fout) {
            if (iter > 0) f = evaluate<W, C>(A, sh, sh.x, sh.g);
            for (int k = tid; k < 3 * N; k += blockDim.x) A.fout[3 * (size_t)o + k] = sh.F[k];
            if (A.uout && tid < 6) A.uout[6 * (size_t)s + tid] = sh.uvir[tid] + (tid < 3 ? sh.scal[4] : 0.0);
            __syncthreads();
        }
        /* results: Cartesian positions of the final DOF vector */
        if (tid == 0) {
            if (rlxt == 3) {
                const double *q = sh.x + 3 * N;
                sh.L[0] = q[0]; sh.L[4] = q[1]; sh.L[8] = q[2]; sh.L[1] = q[3]; sh.L[5] = q[4];
                sh.L[6] = q[5]; sh.L[3] = q[6]; sh.L[7] = q[7]; sh.L[2] = q[8];
            }
            for (int k = 0; k < 9; k++) A.lat[9 * s + k] = sh.L[k];
            A.H[s] = f;
            A.iters[s] = iter;
            A.status[s] = status;
        }
        __syncthreads();
        for (int a = tid; a < N; a += blockDim.x)
            for (int q = 0; q < 3; q++)
                A.x[3 * (size_t)(o + a) + q] = sh.x[3 * a] * sh.L[q] + sh.x[3 * a + 1] * sh.L[3 + q] + sh.x[3 * a + 2] * sh.L[6 + q];
        __syncthreads();
    }
    if constexpr (C > 1) {
        /* queue empty: the exit command, then the last barrier */
        if (tid == 0) sh.cmd_s = -1;
        cooperative_groups::this_cluster().sync();
        cooperative_groups::this_cluster().sync();
    }
    flush_work(A, sh);
}

}  // namespace

/* ---------------- host launcher ---------------- */

static int build_bparams(const mb_model *m, BParams *B, float **w_out, size_t *wlen) {
    const mb_params &P = m->P;
    memset(B, 0, sizeof(*B));
    if (P.ne > BNE || P.nz > BNZ || P.nlam > BNLAM || P.D > BMAXD || P.ng2 > 16) return -1;
    B->nspc = P.nspc; B->D = P.D; B->ng2 = P.ng2; B->ng4 = P.ng4; B->ne = P.ne; B->nz = P.nz; B->nlam = P.nlam;
    B->h1 = P.h1; B->h2 = P.h2;
    memcpy(B->ind2, P.ind2, sizeof(B->ind2));
    memcpy(B->ind4, P.ind4, sizeof(B->ind4));
    for (int p = 0; p < MB_NPAIR; p++) {
        B->f_rc2[p] = (float)P.f_rc2[p];
        B->f_rc4[p] = (float)P.f_rc4[p];
        B->f_rc4sq[p] = (float)P.f_rc4sq[p];
        for (int f = 0; f < MB_MAXG2; f++) {
            B->f_eta2[p][f] = (float)P.f_eta2[p][f];
            B->f_rs[p][f] = (float)P.f_rs[p][f];
        }
        for (int e = 0; e < MB_MAXE; e++) B->f_eta4[p][e] = (float)P.f_eta4[p][e];
    }
    B->d_rc2 = (float)P.d_rc2; B->d_rc4 = (float)P.d_rc4; B->d_rc4sq = (float)P.d_rc4sq;
    for (int f = 0; f < MB_MAXG2; f++) {
        B->d_eta2[f] = (float)P.d_eta2[f];
        B->d_rs[f] = (float)P.d_rs[f];
    }
    for (int e = 0; e < MB_MAXE; e++) B->d_eta4[e] = (float)P.d_eta4[e];
    if (!P.zeta_int) return -1;
    for (int z = 0; z < MB_MAXZ; z++) {
        B->zeta[z] = (float)P.zeta[z];
        B->powz[z] = (float)P.powz[z];
        B->zbits[z] = z < P.nz ? P.zbits[z] : 0;
        B->zstd = P.zeta_std;
        B->zm1bits[z] = z < P.nz ? P.zm1bits[z] : 0;
    }
    for (int l = 0; l < MB_MAXL; l++) B->lam[l] = (float)P.lam[l];
    for (int f = 0; f < P.ng4; f++) B->g4_cell[f] = P.g4_e[f] * BNZL + (P.g4_zl[f] / P.nlam) * BNLAM + P.g4_zl[f] % P.nlam;
    for (int s = 0; s < MB_MAXSPC; s++) {
        B->rm[s] = P.rm[s];
        B->w_off[s] = P.w_off[s];
    }
    B->rc = m->rc_list;
    *wlen = m->weights_len;
    float *w = (float *)malloc(sizeof(float) * m->weights_len);
    for (size_t k = 0; k < m->weights_len; k++) w[k] = (float)m->weights[k];
    *w_out = w;
    return 0;
}

/* launch geometry of k_relax_batch<W, C> on this device: how many CTAs
 * (C = 1) or clusters of C CTAs can be resident at once */
static void cluster_config(cudaLaunchConfig_t *cfg, cudaLaunchAttribute *at, int units, int W, int C, size_t smem,
                           cudaStream_t st) {
    *cfg = cudaLaunchConfig_t{};
    cfg->gridDim = dim3(units * C);
    cfg->blockDim = dim3(W * 32);
    cfg->dynamicSmemBytes = smem;
    cfg->stream = st;
    at->id = cudaLaunchAttributeClusterDimension;
    at->val.clusterDim.x = C;
    at->val.clusterDim.y = 1;
    at->val.clusterDim.z = 1;
    cfg->attrs = at;
    cfg->numAttrs = 1;
}

template <int W, int C>
static cudaError_t batch_config(int sms, int *units) {
    const size_t smem = sizeof(BShared<W>);
    cudaError_t e = cudaFuncSetAttribute(k_relax_batch<W, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (C == 1) {
        int per = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_relax_batch<W, C>, W * 32, smem);
        *units = per * sms;
        return e;
    }
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute at;
    cluster_config(&cfg, &at, 1, W, C, smem, 0);
    return cudaOccupancyMaxActiveClusters(units, k_relax_batch<W, C>, &cfg);
}

template <int W, int C>
static cudaError_t batch_launch(int units, cudaStream_t st, const BArgs &a) {
    if (C == 1) {
        k_relax_batch<W, C><<<units, W * 32, sizeof(BShared<W>), st>>>(a);
        return cudaGetLastError();
    }
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute at;
    cluster_config(&cfg, &at, units, W, C, sizeof(BShared<W>), st);
    return cudaLaunchKernelEx(&cfg, k_relax_batch<W, C>, a);
}

/* Curvature constant of the line search's strong Wolfe test.  The
 * reference's minimiser uses its tolerance, 0.1, which on the EA population
 * costs 3.3 evaluations per BFGS iteration; 0.5 takes 2.1 at the same
 * iteration count and convergence (the minima differ from 0.1's by the
 * spread of FP32 paths), so the batched relax uses 0.5.
 * MAISE_B200_BATCH_SIGMA overrides it with a value in (0, 1). */
static double batch_sigma() {
    const char *e = getenv("MAISE_B200_BATCH_SIGMA");
    if (e) {
        const double v = atof(e);
        if (v > 0.0 && v < 1.0) return v;
    }
    return 0.5;
}

extern "C" int mbk_relax_batch(const mb_model *m, int S, const int *d_nat, const int *d_off, const int *d_spc,
                               const int *d_order, double *d_lat, double *d_x, double p_ev, double urep, int rlxt, int mitr, double fmax,
                               double *d_H, int *d_iters, int *d_status, double *d_frc, double *d_str,
                               void *stream, long long *evals_out, float *ms_out) {
    /* evals_out[4]: evaluations, atom evaluations, pairs, triplets */
    cudaStream_t st = (cudaStream_t)stream;
    BParams hp;
    float *hw = nullptr;
    size_t wlen = 0;
    if (build_bparams(m, &hp, &hw, &wlen)) return (int)cudaErrorInvalidValue;
    int dev = 0, sms = 0, units = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    /* A population that fits the SMs in about two rounds is bound by its
     * slowest BFGS chains: clusters of 4 CTAs (4 SMs) evaluate each structure,
     * cutting a chain's latency about threefold (256 Mg-Ca structures: 0.88 s
     * against 1.60 s).  Larger populations keep one CTA per structure, which
     * has the higher throughput (4096 Cu-Pd-Ag offspring: 2.10 s against
     * 2.48 s with pairs). */
    int wide = 1, csize = S <= 2 * sms ? 4 : 1;
    {
        /* MAISE_B200_BATCH_WARPS=4 selects the narrow CTA and
         * MAISE_B200_BATCH_CLUSTER=1|2|4 the CTAs per structure (A/B timing) */
        const char *fw = getenv("MAISE_B200_BATCH_WARPS"), *fc = getenv("MAISE_B200_BATCH_CLUSTER");
        if (fw) wide = atoi(fw) != 4;
        if (fc) csize = atoi(fc) == 4 ? 4 : atoi(fc) == 2 ? 2 : 1;
        if (!wide) csize = 1;
    }
    cudaError_t e = !wide        ? batch_config<4, 1>(sms, &units)
                    : csize == 4 ? batch_config<BWARPS_WIDE, 4>(sms, &units)
                    : csize == 2 ? batch_config<BWARPS_WIDE, 2>(sms, &units)
                                 : batch_config<BWARPS_WIDE, 1>(sms, &units);
    if (csize > 1 && (e != cudaSuccess || units < 1)) {
        /* clusters of this size cannot be placed (e.g. on a partitioned
         * GPU): one CTA per structure */
        cudaGetLastError();
        csize = 1;
        e = batch_config<BWARPS_WIDE, 1>(sms, &units);
    }
    if (e != cudaSuccess) { free(hw); return (int)e; }
    if (units < 1) { free(hw); return (int)cudaErrorInvalidConfiguration; }
    const int gunits = units < S ? units : S; /* CTAs, or clusters of csize CTAs */
    const int grid = gunits * csize;
    BParams *dp = nullptr;
    float *dw = nullptr;
    double *hm = nullptr;
    float4 *nbd = nullptr;
    int *nbj = nullptr, *queue = nullptr;
    long long *evals = nullptr;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    e = cudaMalloc(&dp, sizeof(BParams));
    if (!e) e = cudaMalloc(&dw, sizeof(float) * wlen);
    if (!e) e = cudaMalloc(&hm, sizeof(double) * (size_t)grid * BMAXDOF * BMAXDOF);
    if (!e) e = cudaMalloc(&nbd, sizeof(float4) * (size_t)grid * BMAXN * BMAXNB);
    if (!e) e = cudaMalloc(&nbj, sizeof(int) * (size_t)grid * BMAXN * BMAXNB);
    if (!e) e = cudaMalloc(&queue, sizeof(int));
    if (!e) e = cudaMalloc(&evals, 4 * sizeof(long long));
    if (!e) e = cudaMemcpyAsync(dp, &hp, sizeof(BParams), cudaMemcpyHostToDevice, st);
    if (!e) e = cudaMemcpyAsync(dw, hw, sizeof(float) * wlen, cudaMemcpyHostToDevice, st);
    if (!e) e = cudaMemsetAsync(queue, 0, sizeof(int), st);
    if (!e) e = cudaMemsetAsync(evals, 0, 4 * sizeof(long long), st);
    if (!e) {
        BArgs a;
        a.S = S; a.rlxt = rlxt; a.mitr = mitr;
        a.p_ev = p_ev; a.urep = urep; a.fmax = fmax; a.sigma = batch_sigma();
        a.nat = d_nat; a.off = d_off; a.spc = d_spc; a.order = d_order;
        a.lat = d_lat; a.x = d_x; a.H = d_H; a.iters = d_iters; a.status = d_status;
        a.fout = d_frc; a.uout = d_str;
        a.P = dp; a.W = dw; a.queue = queue; a.hmat = hm; a.nbd = nbd; a.nbj = nbj; a.evals = evals;
        a.work = (unsigned long long *)(evals + 1);
        cudaEventRecord(e0, st);
        e = !wide        ? batch_launch<4, 1>(gunits, st, a)
            : csize == 4 ? batch_launch<BWARPS_WIDE, 4>(gunits, st, a)
            : csize == 2 ? batch_launch<BWARPS_WIDE, 2>(gunits, st, a)
                         : batch_launch<BWARPS_WIDE, 1>(gunits, st, a);
        cudaEventRecord(e1, st);
        if (!e) e = cudaGetLastError();
    }
    if (!e) e = cudaStreamSynchronize(st);
    if (!e && evals_out) e = cudaMemcpy(evals_out, evals, 4 * sizeof(long long), cudaMemcpyDeviceToHost);
    if (!e && ms_out) cudaEventElapsedTime(ms_out, e0, e1);
    cudaFree(dp); cudaFree(dw); cudaFree(hm); cudaFree(nbd); cudaFree(nbj); cudaFree(queue); cudaFree(evals);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    free(hw);
    return (int)e;
}
