/*
 * mb_rdf.cu -- duplicate detection of the evolutionary search on the GPU:
 * the per-species-pair radial distribution of every member (RDF,
 * src/cell.c:369-417) and the overlaps of all pairs of members (CxC,
 * src/cell.c:419-430) that COMP_CL (src/eutl.c:394-413) combines and
 * RANK_TR (src/emod.c:351-368) compares against its cutoff.
 *
 *   k_rdf_ref   one CTA per structure: every (atom, image) pair within Rmax
 *               with species(j) >= species(i) spreads a Gaussian of width
 *               sigma over the bins within 3 sigma of r, tapered by
 *               cos(pi/2 (x - Rmin)/(Rmax - Rmin)) above Rmin; same-species
 *               blocks halved; optionally scaled to unit length.  The
 *               histogram lives in shared memory (FP64) and is written once.
 *   k_gram      the overlap matrix C = R R^T of the S histograms (a dense
 *               FP64 product of S x S outputs over nbins x npair terms).
 */
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdio.h>
#include <stdlib.h>

#include "../../../include/maise_b200.h"

namespace {

constexpr int RDF_THREADS = 256;

/* Cartesian displacement of j's image (i0,i1,i2) from i, in LIST's
 * operation order (src/cell.c:115-121) */
__device__ __forceinline__ double rdf_disp2(const double *L, const double *xi, const double *xj, int i0, int i1,
                                            int i2) {
    double r = 0.0;
#pragma unroll
    for (int q = 0; q < 3; q++) {
        double x = 0.0;
        x = __dadd_rn(x, __dmul_rn((double)i0, L[q]));
        x = __dadd_rn(x, __dmul_rn((double)i1, L[3 + q]));
        x = __dadd_rn(x, __dmul_rn((double)i2, L[6 + q]));
        x = __dadd_rn(x, __dsub_rn(xj[q], xi[q]));
        r = __dadd_rn(r, __dmul_rn(x, x));
    }
    return r;
}

struct RdfArgs {
    int S, nspc, nbins, ND, normalise;
    const int *off, *spc;
    const double *lat, *x;
    double rmin, rmax, sigma;
    double *out; /* [S][npair][nbins] */
};

__global__ void __launch_bounds__(RDF_THREADS) k_rdf_ref(RdfArgs A) {
    extern __shared__ __align__(16) double hist[]; /* [npair][nbins] */
    __shared__ double L[9], R[9], red[RDF_THREADS / 32];
    __shared__ int nq[3];
    const int s = blockIdx.x, tid = threadIdx.x;
    const int o = A.off[s], N = A.off[s + 1] - o, ns = A.nspc, nb = A.nbins;
    const int npair = ns * (ns + 1) / 2;
    for (int k = tid; k < npair * nb; k += blockDim.x) hist[k] = 0.0;
    if (tid == 0) {
        for (int k = 0; k < 9; k++) L[k] = A.lat[9 * (size_t)s + k];
        R[6] = L[1] * L[5] - L[2] * L[4];
        R[7] = L[2] * L[3] - L[0] * L[5];
        R[8] = L[0] * L[4] - L[1] * L[3];
        R[0] = L[4] * L[8] - L[5] * L[7];
        R[1] = L[5] * L[6] - L[3] * L[8];
        R[2] = L[3] * L[7] - L[4] * L[6];
        R[3] = L[7] * L[2] - L[8] * L[1];
        R[4] = L[8] * L[0] - L[6] * L[2];
        R[5] = L[6] * L[1] - L[7] * L[0];
        const double t = 1.0 / (L[0] * L[4] * L[8] + L[1] * L[5] * L[6] + L[2] * L[3] * L[7] - L[0] * L[5] * L[7] -
                                L[1] * L[3] * L[8] - L[2] * L[4] * L[6]);
        for (int k = 0; k < 9; k++) R[k] *= t;
        for (int q = 0; q < 3; q++) {
            const double len = sqrt(R[3 * q] * R[3 * q] + R[3 * q + 1] * R[3 * q + 1] + R[3 * q + 2] * R[3 * q + 2]);
            nq[q] = q < A.ND ? (int)ceil(A.rmax * len) : 0;
        }
    }
    __syncthreads();
    const double dr = A.rmax / (double)nb, rc2 = A.rmax * A.rmax;
    const int Do = (int)(3.0 * A.sigma / dr);
    const double DRi = 0.5 / (A.sigma * A.sigma);
    const int w0 = 2 * nq[0] + 1, w1 = 2 * nq[1] + 1, w2 = 2 * nq[2] + 1, nimg = w0 * w1 * w2;
    const long long total = (long long)N * N * nimg;
    for (long long c = tid; c < total; c += blockDim.x) {
        const int im = (int)(c % nimg);
        const long long ij = c / nimg;
        const int j = (int)(ij % N), i = (int)(ij / N);
        const int si = A.spc[o + i], sj = A.spc[o + j];
        if (sj < si) continue;
        const int i2 = im % w2 - nq[2], t = im / w2, i1 = t % w1 - nq[1], i0 = t / w1 - nq[0];
        if (i == j && i0 == 0 && i1 == 0 && i2 == 0) continue;
        const double *xi = A.x + 3 * (size_t)(o + i), *xj = A.x + 3 * (size_t)(o + j);
        const double r2 = rdf_disp2(L, xi, xj, i0, i1, i2);
        if (!(r2 < rc2)) continue;
        const double r = sqrt(r2);
        const int ob = (int)(r / dr);
        const int pair = si * ns - si * (si - 1) / 2 + (sj - si); /* (si, sj), si <= sj, row-major */
        double *h = hist + (size_t)pair * nb;
        for (int k = ob - Do; k <= ob + Do; k++) {
            if (k < 0 || k >= nb) continue;
            const double xk = (double)k * dr;
            const double f = xk < A.rmin ? 1.0 : cos(0.5 * CUDART_PI * (xk - A.rmin) / (A.rmax - A.rmin));
            atomicAdd(h + k, f * exp(-(r - xk) * (r - xk) * DRi));
        }
    }
    __syncthreads();
    /* same-species blocks hold each pair twice (i-j and j-i): halved */
    for (int m = 0; m < ns; m++) {
        const int pair = m * ns - m * (m - 1) / 2;
        for (int k = tid; k < nb; k += blockDim.x) hist[(size_t)pair * nb + k] *= 0.5;
    }
    __syncthreads();
    double scale = 1.0;
    if (A.normalise) {
        double ss = 0.0;
        for (int k = tid; k < npair * nb; k += blockDim.x) ss += hist[k] * hist[k];
        for (int off = 16; off > 0; off >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, off);
        if ((tid & 31) == 0) red[tid >> 5] = ss;
        __syncthreads();
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x / 32); w++) tot += red[w];
        scale = tot > 0.0 ? 1.0 / sqrt(tot) : 0.0;
    }
    double *out = A.out + (size_t)s * npair * nb;
    for (int k = tid; k < npair * nb; k += blockDim.x) out[k] = hist[k] * scale;
}

/* C[p][q] = sum_t A[p][t] A[q][t], p, q < S, t < T: 64 x 64 tiles, each
 * thread a 4 x 4 block, the operands staged through shared memory in
 * chunks of 16 terms */
__global__ void __launch_bounds__(256) k_gram(int S, int T, const double *__restrict__ A, double *__restrict__ C) {
    __shared__ double a[16][64 + 1], b[16][64 + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int p0 = blockIdx.y * 64, q0 = blockIdx.x * 64;
    double acc[4][4] = {};
    for (int t0 = 0; t0 < T; t0 += 16) {
        for (int e = threadIdx.x; e < 16 * 64; e += 256) {
            const int r = e / 16, k = e % 16;
            const int p = p0 + r, q = q0 + r, t = t0 + k;
            a[k][r] = (p < S && t < T) ? A[(size_t)p * T + t] : 0.0;
            b[k][r] = (q < S && t < T) ? A[(size_t)q * T + t] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; k++) {
            double av[4], bv[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                av[u] = a[k][ty * 4 + u];
                bv[u] = b[k][tx * 4 + u];
            }
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int v = 0; v < 4; v++) acc[u][v] += av[u] * bv[v];
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const int p = p0 + ty * 4 + u, q = q0 + tx * 4 + v;
            if (p < S && q < S) C[(size_t)p * S + q] = acc[u][v];
        }
}

}  // namespace

extern "C" int mb_handle_fail(int code, const char *msg);

static int rdf_cuda(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return MB_OK;
    static __thread char msg[200];
    snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
    return mb_handle_fail(MB_ERR_CUDA, msg);
}

extern "C" int mb_rdf(int device, int S, const int *nat, const int *atmn, const double *lat, const double *x, int ND,
                      int nspc, int nbins, double rmin, double rmax, double sigma, int normalise, double *rdf) {
    if (S < 1 || !nat || !atmn || !lat || !x || !rdf || nspc < 1 || nspc > 3 || nbins < 1 || !(rmax > 0.0) ||
        !(rmin <= rmax) || !(sigma > 0.0) || ND < 0 || ND > 3)
        return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    const int npair = nspc * (nspc + 1) / 2;
    const size_t smem = sizeof(double) * (size_t)npair * nbins;
    if (smem > 200 * 1024) return mb_handle_fail(MB_ERR_ARG, "nbins x species pairs exceed the shared histogram");
    int *off = (int *)malloc(sizeof(int) * (S + 1));
    off[0] = 0;
    for (int s = 0; s < S; s++) {
        if (nat[s] < 1) {
            free(off);
            return mb_handle_fail(MB_ERR_ARG, "empty structure");
        }
        off[s + 1] = off[s] + nat[s];
    }
    for (int k = 0; k < off[S]; k++)
        if (atmn[k] < 0 || atmn[k] >= nspc) {
            free(off);
            return mb_handle_fail(MB_ERR_ARG, "species index out of range");
        }
    int rc = rdf_cuda(cudaSetDevice(device), "cudaSetDevice");
    int *d_off = nullptr, *d_spc = nullptr;
    double *d_lat = nullptr, *d_x = nullptr, *d_out = nullptr;
    const size_t nout = (size_t)S * npair * nbins;
    if (!rc) rc = rdf_cuda(cudaMalloc(&d_off, sizeof(int) * (S + 1)), "cudaMalloc");
    if (!rc) rc = rdf_cuda(cudaMalloc(&d_spc, sizeof(int) * off[S]), "cudaMalloc");
    if (!rc) rc = rdf_cuda(cudaMalloc(&d_lat, sizeof(double) * 9 * S), "cudaMalloc");
    if (!rc) rc = rdf_cuda(cudaMalloc(&d_x, sizeof(double) * 3 * off[S]), "cudaMalloc");
    if (!rc) rc = rdf_cuda(cudaMalloc(&d_out, sizeof(double) * nout), "cudaMalloc");
    if (!rc) rc = rdf_cuda(cudaMemcpy(d_off, off, sizeof(int) * (S + 1), cudaMemcpyHostToDevice), "H2D");
    if (!rc) rc = rdf_cuda(cudaMemcpy(d_spc, atmn, sizeof(int) * off[S], cudaMemcpyHostToDevice), "H2D");
    if (!rc) rc = rdf_cuda(cudaMemcpy(d_lat, lat, sizeof(double) * 9 * S, cudaMemcpyHostToDevice), "H2D");
    if (!rc) rc = rdf_cuda(cudaMemcpy(d_x, x, sizeof(double) * 3 * off[S], cudaMemcpyHostToDevice), "H2D");
    if (!rc && smem > 48 * 1024)
        rc = rdf_cuda(cudaFuncSetAttribute(k_rdf_ref, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                      "shared-memory opt-in");
    if (!rc) {
        RdfArgs a;
        a.S = S; a.nspc = nspc; a.nbins = nbins; a.ND = ND; a.normalise = normalise ? 1 : 0;
        a.off = d_off; a.spc = d_spc; a.lat = d_lat; a.x = d_x;
        a.rmin = rmin; a.rmax = rmax; a.sigma = sigma; a.out = d_out;
        k_rdf_ref<<<S, RDF_THREADS, smem>>>(a);
        rc = rdf_cuda(cudaGetLastError(), "k_rdf_ref");
    }
    if (!rc) rc = rdf_cuda(cudaMemcpy(rdf, d_out, sizeof(double) * nout, cudaMemcpyDeviceToHost), "D2H");
    cudaFree(d_off); cudaFree(d_spc); cudaFree(d_lat); cudaFree(d_x); cudaFree(d_out);
    free(off);
    return rc;
}

extern "C" int mb_rdf_overlap(int device, int S, int len, const double *rdf, double *cxc) {
    if (S < 1 || len < 1 || !rdf || !cxc) return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    int rc = rdf_cuda(cudaSetDevice(device), "cudaSetDevice");
    double *d_a = nullptr, *d_c = nullptr;
    if (!rc) rc = rdf_cuda(cudaMalloc(&d_a, sizeof(double) * (size_t)S * len), "cudaMalloc");
    if (!rc) rc = rdf_cuda(cudaMalloc(&d_c, sizeof(double) * (size_t)S * S), "cudaMalloc");
    if (!rc) rc = rdf_cuda(cudaMemcpy(d_a, rdf, sizeof(double) * (size_t)S * len, cudaMemcpyHostToDevice), "H2D");
    if (!rc) {
        k_gram<<<dim3((S + 63) / 64, (S + 63) / 64), 256>>>(S, len, d_a, d_c);
        rc = rdf_cuda(cudaGetLastError(), "k_gram");
    }
    if (!rc) rc = rdf_cuda(cudaMemcpy(cxc, d_c, sizeof(double) * (size_t)S * S, cudaMemcpyDeviceToHost), "D2H");
    cudaFree(d_a);
    cudaFree(d_c);
    return rc;
}
