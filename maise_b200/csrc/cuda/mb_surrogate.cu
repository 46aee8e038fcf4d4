/*
 * mb_surrogate.cu -- kernels of the surrogate screen for EA offspring.
 *
 * The screen ranks unrelaxed offspring by a predicted relaxed enthalpy per
 * atom so that only the best fraction goes on to a full relaxation.  Its
 * input is a per-species-pair radial histogram (the analogue of RDF,
 * src/cell.c:369-417, at 128 bins); its model is a small FP32 MLP
 * (nin -> 128 -> 64 -> 64 -> 1, SiLU) trained with Adam on
 * unrelaxed -> relaxed pairs.  Nothing here exists in the reference, which
 * relaxes every offspring.
 *
 * Kernels:
 *   k_rdf       one CTA per structure: fractional coordinates in shared
 *               memory, every (i, j, image) within rmax deposits a tapered
 *               Gaussian into a shared histogram (FP64 distances and
 *               weights, FP32 shared atomics); writes the histogram / N.
 *   k_gemm      64x64x16 register-tiled FP32 GEMM, C = op(A) op(B), with
 *               fused epilogues: bias + SiLU (keeping the pre-activation),
 *               bias only, plain store, and product with SiLU'(Z) for the
 *               backward pass.  The layers are at most 4096 x 768 x 128,
 *               FP32 by specification, so SIMT FMA tiles are used.
 *   k_colsum    bias gradients (column sums of dZ).
 *   k_mse       squared-error loss and its gradient for one batch.
 *   k_adam      Adam update of the flat parameter vector.
 *   k_gather    minibatch rows by index, standardised on the fly.
 *   k_colstats  per-feature mean and 1/std of the training features.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../host/mb_surrogate_k.h"

/* ------------------------------------------------------------ histogram */

__global__ void __launch_bounds__(256) k_rdf(int S, const int *__restrict__ off, const int *__restrict__ spc,
                                            const double *__restrict__ lat, const double *__restrict__ x, int nspc,
                                            int nbins, double rmax, double sigma, float *__restrict__ feat,
                                            int *__restrict__ status) {
    extern __shared__ float hist[];
    __shared__ double L[9], Li[9];
    __shared__ double fr[3 * SUR_MAX_ATOMS];
    __shared__ int sp[SUR_MAX_ATOMS];
    __shared__ int nimg[3];
    __shared__ int bad;
    const int s = blockIdx.x, tid = threadIdx.x, bd = blockDim.x;
    if (s >= S) return;
    const int a0 = off[s], N = off[s + 1] - a0;
    const int P = nspc * (nspc + 1) / 2;
    for (int k = tid; k < P * nbins; k += bd) hist[k] = 0.0f;
    if (tid < 9) L[tid] = lat[9 * s + tid];
    __syncthreads();
    if (tid == 0) {
        /* inverse of the row-vector lattice by cofactors */
        const double c00 = L[4] * L[8] - L[5] * L[7], c01 = L[5] * L[6] - L[3] * L[8], c02 = L[3] * L[7] - L[4] * L[6];
        const double det = L[0] * c00 + L[1] * c01 + L[2] * c02;
        const double id = 1.0 / det;
        Li[0] = c00 * id;
        Li[3] = c01 * id;
        Li[6] = c02 * id;
        Li[1] = (L[2] * L[7] - L[1] * L[8]) * id;
        Li[4] = (L[0] * L[8] - L[2] * L[6]) * id;
        Li[7] = (L[1] * L[6] - L[0] * L[7]) * id;
        Li[2] = (L[1] * L[5] - L[2] * L[4]) * id;
        Li[5] = (L[2] * L[3] - L[0] * L[5]) * id;
        Li[8] = (L[0] * L[4] - L[1] * L[3]) * id;
        /* images needed along each lattice vector: rmax over the plane
         * spacing, plus half a cell for the minimum-image fractional shift */
        const double V = fabs(det);
        bad = (N < 1 || N > SUR_MAX_ATOMS || !(V > 0.0));
        for (int a = 0; a < 3; a++) {
            const double *b = L + 3 * ((a + 1) % 3), *c = L + 3 * ((a + 2) % 3);
            const double cx = b[1] * c[2] - b[2] * c[1], cy = b[2] * c[0] - b[0] * c[2], cz = b[0] * c[1] - b[1] * c[0];
            const double h = V / sqrt(cx * cx + cy * cy + cz * cz);
            const double n = ceil(rmax / h + 0.5);
            if (!(n <= SUR_MAX_IMG)) bad = 1;
            nimg[a] = bad ? 0 : (int)n;
        }
    }
    __syncthreads();
    if (bad) {
        if (tid == 0) atomicOr(status, 1);
        for (int k = tid; k < P * nbins; k += bd) feat[(size_t)s * P * nbins + k] = 0.0f;
        return;
    }
    for (int i = tid; i < N; i += bd) {
        const double *xi = x + 3 * (size_t)(a0 + i);
        for (int c = 0; c < 3; c++) fr[3 * i + c] = xi[0] * Li[c] + xi[1] * Li[3 + c] + xi[2] * Li[6 + c];
        sp[i] = spc[a0 + i];
    }
    __syncthreads();
    const double dr = rmax / nbins;
    const int Do = (int)(3.0 * sigma / dr);
    const double DR = 0.5 / (sigma * sigma);
    const double rc2 = rmax * rmax;
    const int n0 = nimg[0], n1 = nimg[1], n2 = nimg[2];
    for (int w = tid; w < N * N; w += bd) {
        const int i = w / N, j = w - i * N;
        const int si = sp[i], sj = sp[j];
        if (sj < si) continue;
        const int p = si * nspc - si * (si - 1) / 2 + (sj - si);
        double d[3];
        for (int c = 0; c < 3; c++) {
            const double t = fr[3 * j + c] - fr[3 * i + c];
            d[c] = t - rint(t);
        }
        for (int ta = -n0; ta <= n0; ta++)
            for (int tb = -n1; tb <= n1; tb++)
                for (int tc = -n2; tc <= n2; tc++) {
                    const double u0 = d[0] + ta, u1 = d[1] + tb, u2 = d[2] + tc;
                    const double vx = u0 * L[0] + u1 * L[3] + u2 * L[6];
                    const double vy = u0 * L[1] + u1 * L[4] + u2 * L[7];
                    const double vz = u0 * L[2] + u1 * L[5] + u2 * L[8];
                    const double r2 = vx * vx + vy * vy + vz * vz;
                    if (!(r2 < rc2) || r2 == 0.0) continue;
                    const double r = sqrt(r2);
                    const int o = (int)(r / dr);
                    for (int k = o - Do; k <= o + Do; k++) {
                        if (k < 0 || k >= nbins) continue;
                        const double xk = k * dr;
                        const double f = cos(0.5 * M_PI * xk / rmax) * exp(-(r - xk) * (r - xk) * DR);
                        atomicAdd(&hist[p * nbins + k], (float)f);
                    }
                }
    }
    __syncthreads();
    const float invN = 1.0f / (float)N;
    for (int k = tid; k < P * nbins; k += bd) {
        const int p = k / nbins;
        int diag = 0;
        for (int m = 0; m < nspc; m++) diag |= (p == m * nspc - m * (m - 1) / 2);
        feat[(size_t)s * P * nbins + k] = hist[k] * (diag ? 0.5f : 1.0f) * invN;
    }
}

/* ----------------------------------------------------------------- GEMM */

#define GB_M 64
#define GB_N 64
#define GB_K 16

__device__ __forceinline__ float silu_f(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float dsilu_f(float z) {
    const float s = 1.0f / (1.0f + expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

/* C[m, n] = sum_k A(m, k) B(k, n), A(m, k) = TA ? A[k lda + m] : A[m lda + k],
 * B(k, n) = TB ? B[n ldb + k] : B[k ldb + n]; row-major C with leading
 * dimension ldc; EP selects the epilogue (SUR_EP_*). */
template <bool TA, bool TB, int EP>
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, const float *__restrict__ A, int lda,
                                             const float *__restrict__ B, int ldb, float *__restrict__ C, int ldc,
                                             const float *__restrict__ bias, float *__restrict__ Z,
                                             const float *__restrict__ Zp) {
    __shared__ float As[GB_K][GB_M + 4];
    __shared__ float Bs[GB_K][GB_N + 4];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int m0 = blockIdx.y * GB_M, n0 = blockIdx.x * GB_N;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0f;
    for (int k0 = 0; k0 < K; k0 += GB_K) {
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int e = tid + 256 * r;
            int m, k;
            if (TA) {
                m = e % GB_M;
                k = e / GB_M;
            } else {
                k = e % GB_K;
                m = e / GB_K;
            }
            const int gm = m0 + m, gk = k0 + k;
            float v = 0.0f;
            if (gm < M && gk < K) v = TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
            As[k][m] = v;
        }
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int e = tid + 256 * r;
            int n, k;
            if (TB) {
                k = e % GB_K;
                n = e / GB_K;
            } else {
                n = e % GB_N;
                k = e / GB_N;
            }
            const int gn = n0 + n, gk = k0 + k;
            float v = 0.0f;
            if (gn < N && gk < K) v = TB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn];
            Bs[k][n] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GB_K; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int gm = m0 + ty * 4 + i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int gn = n0 + tx * 4 + j;
            if (gn >= N) continue;
            const size_t o = (size_t)gm * ldc + gn;
            float v = acc[i][j];
            if (EP == SUR_EP_BIAS_SILU) {
                v += bias[gn];
                Z[o] = v;
                C[o] = silu_f(v);
            } else if (EP == SUR_EP_BIAS) {
                C[o] = v + bias[gn];
            } else if (EP == SUR_EP_DSILU) {
                C[o] = v * dsilu_f(Zp[o]);
            } else {
                C[o] = v;
            }
        }
    }
}

extern "C" int surk_gemm(int ta, int tb, int ep, int M, int N, int K, const float *A, int lda, const float *B, int ldb,
                         float *C, int ldc, const float *bias, float *Z, const float *Zp, void *stream) {
    dim3 grid((N + GB_N - 1) / GB_N, (M + GB_M - 1) / GB_M);
    cudaStream_t st = (cudaStream_t)stream;
#define SUR_GEMM(TA_, TB_, EP_) k_gemm<TA_, TB_, EP_><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, Z, Zp)
    if (!ta && tb && ep == SUR_EP_BIAS_SILU) SUR_GEMM(false, true, SUR_EP_BIAS_SILU);
    else if (!ta && tb && ep == SUR_EP_BIAS) SUR_GEMM(false, true, SUR_EP_BIAS);
    else if (!ta && !tb && ep == SUR_EP_DSILU) SUR_GEMM(false, false, SUR_EP_DSILU);
    else if (ta && !tb && ep == SUR_EP_STORE) SUR_GEMM(true, false, SUR_EP_STORE);
    else return (int)cudaErrorInvalidValue;
#undef SUR_GEMM
    return (int)cudaGetLastError();
}

/* ------------------------------------------------------- small kernels */

__global__ void k_colsum(int B, int O, const float *__restrict__ dZ, float *__restrict__ out) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= O) return;
    float s = 0.0f;
    for (int b = 0; b < B; b++) s += dZ[(size_t)b * O + o];
    out[o] = s;
}

__global__ void __launch_bounds__(256) k_mse(int B, const float *__restrict__ y, const float *__restrict__ t,
                                            float *__restrict__ dy, double *__restrict__ loss) {
    __shared__ double red[256];
    double s = 0.0;
    for (int b = threadIdx.x; b < B; b += blockDim.x) {
        const float e = y[b] - t[b];
        dy[b] = 2.0f * e / (float)B;
        s += (double)e * e;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = red[0] / B;
}

__global__ void k_adam(long n, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const float gk = g[k];
        const float mk = b1 * m[k] + (1.0f - b1) * gk;
        const float vk = b2 * v[k] + (1.0f - b2) * gk * gk;
        m[k] = mk;
        v[k] = vk;
        p[k] -= lr * (mk * c1) / (sqrtf(vk * c2) + eps);
    }
}

__global__ void k_gather(int B, int F, const int *__restrict__ idx, const float *__restrict__ X,
                         const float *__restrict__ mean, const float *__restrict__ istd, float *__restrict__ out,
                         const float *__restrict__ T, float tmean, float tistd, float *__restrict__ tout) {
    const int b = blockIdx.x;
    if (b >= B) return;
    const long r = idx ? idx[b] : b;
    const float *src = X + (size_t)r * F;
    float *dst = out + (size_t)b * F;
    for (int f = threadIdx.x; f < F; f += blockDim.x) dst[f] = (src[f] - mean[f]) * istd[f];
    if (T && threadIdx.x == 0) tout[b] = (T[r] - tmean) * tistd;
}

__global__ void k_colstats(int S, int F, const float *__restrict__ X, float *__restrict__ mean,
                           float *__restrict__ istd) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    double s = 0.0;
    for (int r = 0; r < S; r++) s += X[(size_t)r * F + f];
    const double mu = s / S;
    double q = 0.0;
    for (int r = 0; r < S; r++) {
        const double e = X[(size_t)r * F + f] - mu;
        q += e * e;
    }
    mean[f] = (float)mu;
    istd[f] = (float)(1.0 / sqrt(q / S + SUR_VAR_FLOOR));
}

/* ------------------------------------------------------------ launchers */

extern "C" int surk_rdf(int S, const int *off, const int *spc, const double *lat, const double *x, int nspc, int nbins,
                        double rmax, double sigma, float *feat, int *status, void *stream) {
    const int P = nspc * (nspc + 1) / 2;
    const size_t smem = sizeof(float) * P * nbins;
    if (nspc < 1 || nspc > SUR_MAX_SPC || nbins < 1 || smem > 48 * 1024) return (int)cudaErrorInvalidValue;
    k_rdf<<<S, 256, smem, (cudaStream_t)stream>>>(S, off, spc, lat, x, nspc, nbins, rmax, sigma, feat, status);
    return (int)cudaGetLastError();
}

extern "C" int surk_colsum(int B, int O, const float *dZ, float *out, void *stream) {
    k_colsum<<<(O + 127) / 128, 128, 0, (cudaStream_t)stream>>>(B, O, dZ, out);
    return (int)cudaGetLastError();
}

extern "C" int surk_mse(int B, const float *y, const float *t, float *dy, double *loss, void *stream) {
    k_mse<<<1, 256, 0, (cudaStream_t)stream>>>(B, y, t, dy, loss);
    return (int)cudaGetLastError();
}

extern "C" int surk_adam(long n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2, float eps,
                         float c1, float c2, void *stream) {
    long blocks = (n + 255) / 256;
    if (blocks > 1184) blocks = 1184; /* 148 SMs x 8 */
    k_adam<<<(int)blocks, 256, 0, (cudaStream_t)stream>>>(n, p, g, m, v, lr, b1, b2, eps, c1, c2);
    return (int)cudaGetLastError();
}

extern "C" int surk_gather(int B, int F, const int *idx, const float *X, const float *mean, const float *istd,
                           float *out, const float *T, float tmean, float tistd, float *tout, void *stream) {
    if (B < 1) return 0;
    k_gather<<<B, 256, 0, (cudaStream_t)stream>>>(B, F, idx, X, mean, istd, out, T, tmean, tistd, tout);
    return (int)cudaGetLastError();
}

extern "C" int surk_colstats(int S, int F, const float *X, float *mean, float *istd, void *stream) {
    k_colstats<<<(F + 127) / 128, 128, 0, (cudaStream_t)stream>>>(S, F, X, mean, istd);
    return (int)cudaGetLastError();
}
