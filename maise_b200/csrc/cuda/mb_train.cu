/*
 * mb_train.cu -- training of the per-species MLP on the GPU: the objective
 * and gradient of MAISE's network training (tot_err_gsl / dfunc_gsl,
 * src/nmin.c:93-305, with the energy back-propagation of DE_ANN_PARA,
 * src/nmlp.c:292-354, and the force terms of FRC_ANN_PARA / DF_ANN_PARA,
 * src/nmlp.c:29-290), minimised by the project BFGS (mb_bfgs.c) as MLP_MIN
 * does with GSL's vector_bfgs2 (src/nmin.c:314-445).
 *
 * Objective over S training structures with reference energies E_s,
 * weights w_s and atoms N_s, and (force training, EFS 1 or 3) marked atoms
 * i with reference forces F_i:
 *   RT = (WE sum_s w_s ((E_s - E(s)) / N_s)^2
 *         + WF sum_s w_s sum_{i marked} |F_i - f_i|^2) / S
 *        + LREG sum(b^2 + W^2),
 *   E(s) = sum over the structure's atoms of the species network on the
 *   scaled inputs x = (G - Rmin) DR,
 *   f_i = -sum_b sum_l Fn_b[l] g_o(b)[l], over i's derivative blocks b
 *   (dG_o/dx_i of owner atom o, self block included), g_o = dE_o/dx_o,
 * and its gradient, / S, plus 2 LREG V.  The energy part back-propagates
 * c_s = 2 WE w_s (E(s) - E_s) / N_s^2 through every atom.  The force part
 * is the exact derivative DF_ANN_PARA forms: with dfq = 2 WF w_s (f_i - F_i)
 * and, per block, xn[n] = dfq . (W0 Fn_b)[n] (per axis), xm = W1 diag(d1) xn,
 * beta = W1^T diag(W2 c2) xm, the first-layer weights receive
 * -(ad1 (x) phi_b + gamma_b (x) x_o), phi_b = Fn_b dfq, ad1 = dE/d(layer-1
 * pre-activation), gamma = ad1/d1 c1 xn + d1 beta (summed over axes), and
 * the other layers the terms written in k_tr_fown.
 *
 * Parameters in the reference's V2W order (src/nmlp.c:591-608): per species
 * the biases of all layers (b0[h1], b1[h2], b2), then the weights
 * W0[h1][D], W1[h2][h1], W2[h2].  Hidden layers tanh, output linear.
 *
 * Kernels (FP64; every sum in a fixed order, so results are reproducible):
 *   k_tr_fwd     one warp per atom: hidden activations and the atom energy
 *   k_tr_struct  one thread per structure: E(s), c_s and the loss term
 *   k_tr_delta   one thread per atom: back-propagated deltas
 *   k_tr_ad1     one thread per atom: dE/d(layer-1 pre-activation)
 *   k_tr_fproj   one CTA per block: W0 Fn_b (h1 x 3)
 *   k_tr_frc     one warp per marked atom: f_i, dfq and the force loss term
 *   k_tr_fown    one CTA per block owner: the force-gradient terms of the
 *                owner's network, summed over its blocks in block order
 *   k_tr_grad    one thread per parameter: the sum over the atoms of its
 *                species in atom order, / S, + 2 LREG V
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../../include/maise_train.h"
#include "../host/mb_bfgs.h"

extern "C" int mb_handle_fail(int code, const char *msg);

namespace {

struct TrainDims {
    int S, Na, D, h1, h2, nspc, P; /* P parameters per species */
    double WE, LREG;
};

__host__ __device__ inline int off_b1(const TrainDims &t) { return t.h1; }
__host__ __device__ inline int off_b2(const TrainDims &t) { return t.h1 + t.h2; }
__host__ __device__ inline int off_W0(const TrainDims &t) { return t.h1 + t.h2 + 1; }
__host__ __device__ inline int off_W1(const TrainDims &t) { return off_W0(t) + t.h1 * t.D; }
__host__ __device__ inline int off_W2(const TrainDims &t) { return off_W1(t) + t.h2 * t.h1; }

__global__ void k_tr_fwd(TrainDims t, const double *__restrict__ X, const int *__restrict__ spc,
                         const double *__restrict__ V, double *__restrict__ H1, double *__restrict__ H2,
                         double *__restrict__ Eat) {
    const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= t.Na) return;
    const double *v = V + (size_t)spc[a] * t.P, *x = X + (size_t)a * t.D;
    const double *W0 = v + off_W0(t), *b0 = v;
    double h1[MB_TRAIN_MAXH];
    for (int k = 0; k < t.h1; k++) {
        double acc = 0.0;
        for (int n = lane; n < t.D; n += 32) acc += W0[(size_t)k * t.D + n] * x[n];
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        h1[k] = tanh(b0[k] + acc);
    }
    if (lane == 0) {
        const double *W1 = v + off_W1(t), *b1 = v + off_b1(t), *W2 = v + off_W2(t), *b2 = v + off_b2(t);
        double e = b2[0];
        for (int m = 0; m < t.h2; m++) {
            double s = b1[m];
            for (int k = 0; k < t.h1; k++) s += W1[m * t.h1 + k] * h1[k];
            const double h = tanh(s);
            H2[(size_t)a * t.h2 + m] = h;
            e += W2[m] * h;
        }
        for (int k = 0; k < t.h1; k++) H1[(size_t)a * t.h1 + k] = h1[k];
        Eat[a] = e;
    }
}

__global__ void k_tr_struct(TrainDims t, const int *__restrict__ soff, const double *__restrict__ Eat,
                            const double *__restrict__ Eref, const double *__restrict__ wt, double *__restrict__ Es,
                            double *__restrict__ cs, double *__restrict__ ls) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= t.S) return;
    double e = 0.0;
    for (int a = soff[s]; a < soff[s + 1]; a++) e += Eat[a];
    const double n = (double)(soff[s + 1] - soff[s]);
    Es[s] = e;
    cs[s] = 2.0 * (e - Eref[s]) / (n * n) * t.WE * wt[s];
    const double r = (Eref[s] - e) / n;
    ls[s] = r * r * wt[s];
}

__global__ void k_tr_delta(TrainDims t, const int *__restrict__ spc, const int *__restrict__ sat,
                           const double *__restrict__ V, const double *__restrict__ H1, const double *__restrict__ H2,
                           const double *__restrict__ cs, double *__restrict__ d0, double *__restrict__ d1,
                           double *__restrict__ ca) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= t.Na) return;
    const double *v = V + (size_t)spc[a] * t.P, *W1 = v + off_W1(t), *W2 = v + off_W2(t);
    const double c = cs[sat[a]];
    ca[a] = c;
    double dl1[MB_TRAIN_MAXH];
    for (int m = 0; m < t.h2; m++) {
        const double h = H2[(size_t)a * t.h2 + m];
        dl1[m] = c * W2[m] * (1.0 - h * h);
        d1[(size_t)a * t.h2 + m] = dl1[m];
    }
    for (int k = 0; k < t.h1; k++) {
        double g = 0.0;
        for (int m = 0; m < t.h2; m++) g += dl1[m] * W1[m * t.h1 + k];
        const double h = H1[(size_t)a * t.h1 + k];
        d0[(size_t)a * t.h1 + k] = g * (1.0 - h * h);
    }
}

/* ---- force training ---- */

/* per atom: ad1[n] = dE/d(pre-activation n of the first hidden layer)
 * = (sum_m W2[m] (1 - e2[m]^2) W1[m][n]) (1 - e1[n]^2) */
__global__ void k_tr_ad1(TrainDims t, const int *__restrict__ spc, const double *__restrict__ V,
                         const double *__restrict__ H1, const double *__restrict__ H2, double *__restrict__ AD1) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= t.Na) return;
    const double *v = V + (size_t)spc[a] * t.P, *W1 = v + off_W1(t), *W2 = v + off_W2(t);
    for (int n = 0; n < t.h1; n++) {
        double al = 0.0;
        for (int m = 0; m < t.h2; m++) {
            const double h = H2[(size_t)a * t.h2 + m];
            al += W2[m] * (1.0 - h * h) * W1[m * t.h1 + n];
        }
        const double e = H1[(size_t)a * t.h1 + n];
        AD1[(size_t)a * t.h1 + n] = al * (1.0 - e * e);
    }
}

/* one CTA per block b: Pj[b][n][q] = sum_l W0[n][l] Fn_b[l][q] with the
 * first-layer weights of the block owner's species */
__global__ void k_tr_fproj(TrainDims t, int NB, const int *__restrict__ bown, const int *__restrict__ spc,
                           const double *__restrict__ V, const double *__restrict__ Fn, double *__restrict__ Pj) {
    const int b = blockIdx.x;
    if (b >= NB) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const double *W0 = V + (size_t)spc[bown[b]] * t.P + off_W0(t);
    const double *fb = Fn + (size_t)b * t.D * 3;
    for (int n = warp; n < t.h1; n += nw) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (int l = lane; l < t.D; l += 32) {
            const double w = W0[(size_t)n * t.D + l];
            a0 += w * fb[3 * l];
            a1 += w * fb[3 * l + 1];
            a2 += w * fb[3 * l + 2];
        }
        for (int o = 16; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        }
        if (lane == 0) {
            double *p = Pj + ((size_t)b * t.h1 + n) * 3;
            p[0] = a0;
            p[1] = a1;
            p[2] = a2;
        }
    }
}

/* one warp per marked atom i: f_i = -sum_b sum_n AD1[o_b][n] Pj[b][n]
 * (FRC_ANN_PARA, src/nmlp.c:53-99), dL/df_i = 2 WF w_s (f_i - F_i)
 * (src/nmlp.c:176-178) and the loss term w_s |F_i - f_i|^2
 * (src/nmin.c:123-127) */
__global__ void k_tr_frc(TrainDims t, int NF, const int *__restrict__ fatom, const int *__restrict__ boff,
                         const int *__restrict__ bown, const int *__restrict__ sat, const double *__restrict__ wt,
                         const double *__restrict__ Fref, const double *__restrict__ AD1,
                         const double *__restrict__ Pj, double WF, double *__restrict__ fpred,
                         double *__restrict__ dfq, double *__restrict__ lf) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= NF) return;
    double f0 = 0.0, f1 = 0.0, f2 = 0.0;
    for (int b = boff[i] + lane; b < boff[i + 1]; b += 32) {
        const double *ad = AD1 + (size_t)bown[b] * t.h1, *p = Pj + (size_t)b * t.h1 * 3;
        for (int n = 0; n < t.h1; n++) {
            f0 += ad[n] * p[3 * n];
            f1 += ad[n] * p[3 * n + 1];
            f2 += ad[n] * p[3 * n + 2];
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        f0 += __shfl_xor_sync(0xffffffffu, f0, o);
        f1 += __shfl_xor_sync(0xffffffffu, f1, o);
        f2 += __shfl_xor_sync(0xffffffffu, f2, o);
    }
    if (lane == 0) {
        const double w = wt[sat[fatom[i]]], f[3] = {-f0, -f1, -f2};
        double l = 0.0;
        for (int q = 0; q < 3; q++) {
            const double r = f[q] - Fref[3 * i + q];
            fpred[3 * i + q] = f[q];
            dfq[3 * i + q] = 2.0 * r * WF * w;
            l += r * r;
        }
        lf[i] = l * w;
    }
}

/* One CTA per block owner o (an atom that is a neighbour, or the marked
 * atom itself, in some marked atom's blocks): the force-gradient terms of
 * DF_ANN_PARA (src/nmlp.c:171-288) for o's network, summed over o's blocks
 * in block order.  Per block b of marked atom i (dfq = dfq_i):
 *   xn[n][q] = dfq[q] Pj[b][n][q]            phi[l] = sum_q Fn_b[l][q] dfq[q]
 *   xm[m][q] = sum_n W1[m][n] d1[n] xn[n][q]
 *   beta[n][q] = sum_m W2[m] c2[m] W1[m][n] xm[m][q]
 *   gamma[n] = sum_q (alpha[n] c1[n] xn[n][q] + d1[n] beta[n][q])
 *   b1[m] -= sum_q W2[m] c2[m] xm[m][q]      W2[m] -= sum_q d2[m] xm[m][q]
 *   W1[m][n] -= sum_q (W2[m] d2[m] d1[n] xn[n][q] + W2[m] c2[m] e1[n] xm[m][q])
 * with e, d = 1 - e^2, c = 2 e (e^2 - 1) of o's activations (GP, GPp, GPc,
 * src/nmlp.c:8-27) and alpha[n] = sum_m W2[m] d2[m] W1[m][n].  Phi and Gam
 * receive sum_b phi and sum_b gamma; the first-layer terms
 * -(ad1 (x) phi + gamma (x) x_o) and b0 -= gamma are formed in k_tr_grad. */
__global__ void __launch_bounds__(128) k_tr_fown(TrainDims t, const int *__restrict__ owners,
                                                 const int *__restrict__ ooff, const int *__restrict__ olist,
                                                 const int *__restrict__ bmk, const int *__restrict__ spc,
                                                 const double *__restrict__ V, const double *__restrict__ H1,
                                                 const double *__restrict__ H2, const double *__restrict__ Fn,
                                                 const double *__restrict__ Pj, const double *__restrict__ dfq,
                                                 double *__restrict__ Phi, double *__restrict__ Gam,
                                                 double *__restrict__ fB1, double *__restrict__ fW1,
                                                 double *__restrict__ fW2) {
    constexpr int H = MB_TRAIN_MAXH;
    __shared__ double e1[H], d1[H], c1[H], al[H], d2[H], c2[H], xn[3 * H], xm[3 * H];
    __shared__ double gam[H], b1a[H], w2a[H], w1a[H * H];
    extern __shared__ double phi[]; /* [D] */
    const int o = owners[blockIdx.x], tid = threadIdx.x, NT = blockDim.x;
    const int h1 = t.h1, h2 = t.h2, D = t.D;
    const double *v = V + (size_t)spc[o] * t.P, *W1 = v + off_W1(t), *W2 = v + off_W2(t);
    if (tid < h1) {
        const double e = H1[(size_t)o * h1 + tid];
        e1[tid] = e;
        d1[tid] = 1.0 - e * e;
        c1[tid] = 2.0 * e * (e * e - 1.0);
        gam[tid] = 0.0;
    }
    if (tid < h2) {
        const double e = H2[(size_t)o * h2 + tid];
        d2[tid] = 1.0 - e * e;
        c2[tid] = 2.0 * e * (e * e - 1.0);
        b1a[tid] = 0.0;
        w2a[tid] = 0.0;
    }
    for (int k = tid; k < h1 * h2; k += NT) w1a[k] = 0.0;
    for (int l = tid; l < D; l += NT) phi[l] = 0.0;
    __syncthreads();
    if (tid < h1) {
        double s = 0.0;
        for (int m = 0; m < h2; m++) s += W2[m] * d2[m] * W1[m * h1 + tid];
        al[tid] = s;
    }
    __syncthreads();
    for (int k = ooff[blockIdx.x]; k < ooff[blockIdx.x + 1]; k++) {
        const int b = olist[k];
        const double *dq = dfq + 3 * (size_t)bmk[b], *fb = Fn + (size_t)b * D * 3;
        const double q0 = dq[0], q1 = dq[1], q2 = dq[2];
        if (tid < 3 * h1) xn[tid] = dq[tid % 3] * Pj[(size_t)b * h1 * 3 + tid];
        for (int l = tid; l < D; l += NT) phi[l] += fb[3 * l] * q0 + fb[3 * l + 1] * q1 + fb[3 * l + 2] * q2;
        __syncthreads();
        if (tid < 3 * h2) {
            const int m = tid / 3, q = tid % 3;
            double s = 0.0;
            for (int n = 0; n < h1; n++) s += W1[m * h1 + n] * d1[n] * xn[3 * n + q];
            xm[tid] = s;
        }
        __syncthreads();
        if (tid < h1) {
            const int n = tid;
            double g = 0.0;
            for (int q = 0; q < 3; q++) {
                double be = 0.0;
                for (int m = 0; m < h2; m++) be += W2[m] * c2[m] * W1[m * h1 + n] * xm[3 * m + q];
                g += al[n] * c1[n] * xn[3 * n + q] + d1[n] * be;
            }
            gam[n] += g;
        } else if (tid < h1 + h2) {
            const int m = tid - h1;
            const double xs = xm[3 * m] + xm[3 * m + 1] + xm[3 * m + 2];
            b1a[m] -= W2[m] * c2[m] * xs;
            w2a[m] -= d2[m] * xs;
        }
        for (int k2 = tid; k2 < h1 * h2; k2 += NT) {
            const int m = k2 / h1, n = k2 % h1;
            double s = 0.0;
            for (int q = 0; q < 3; q++)
                s += W2[m] * d2[m] * d1[n] * xn[3 * n + q] + W2[m] * c2[m] * e1[n] * xm[3 * m + q];
            w1a[k2] -= s;
        }
        __syncthreads();
    }
    for (int l = tid; l < D; l += NT) Phi[(size_t)o * D + l] = phi[l];
    if (tid < h1) Gam[(size_t)o * h1 + tid] = gam[tid];
    if (tid < h2) {
        fB1[(size_t)o * h2 + tid] = b1a[tid];
        fW2[(size_t)o * h2 + tid] = w2a[tid];
    }
    for (int k = tid; k < h1 * h2; k += NT) fW1[(size_t)o * h1 * h2 + k] = w1a[k];
}

/* force-gradient accumulators per atom (all NULL without force training) */
struct ForceTerms {
    const double *AD1, *Phi, *Gam, *fB1, *fW1, *fW2;
};

/* one thread per parameter of one species: the sum over that species'
 * atoms (in atom order) of the parameter's back-propagated terms, energy
 * and (with force training) force */
__global__ void k_tr_grad(TrainDims t, const int *__restrict__ satoms, const int *__restrict__ soffs,
                          const double *__restrict__ X, const double *__restrict__ H1, const double *__restrict__ H2,
                          const double *__restrict__ d0, const double *__restrict__ d1, const double *__restrict__ ca,
                          ForceTerms ft, const double *__restrict__ V, double *__restrict__ grad) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= t.nspc * t.P) return;
    const int s = idx / t.P, p = idx % t.P;
    const int lo = soffs[s], hi = soffs[s + 1];
    const bool F = ft.Gam != nullptr;
    double acc = 0.0;
    if (p < off_b1(t)) {
        const int k = p;
        for (int q = lo; q < hi; q++) {
            const int a = satoms[q];
            acc += d0[(size_t)a * t.h1 + k];
            if (F) acc -= ft.Gam[(size_t)a * t.h1 + k];
        }
    } else if (p < off_b2(t)) {
        const int m = p - off_b1(t);
        for (int q = lo; q < hi; q++) {
            const int a = satoms[q];
            acc += d1[(size_t)a * t.h2 + m];
            if (F) acc += ft.fB1[(size_t)a * t.h2 + m];
        }
    } else if (p < off_W0(t)) {
        for (int q = lo; q < hi; q++) acc += ca[satoms[q]];
    } else if (p < off_W1(t)) {
        const int k = (p - off_W0(t)) / t.D, n = (p - off_W0(t)) % t.D;
        for (int q = lo; q < hi; q++) {
            const int a = satoms[q];
            double dk = d0[(size_t)a * t.h1 + k];
            if (F) {
                dk -= ft.Gam[(size_t)a * t.h1 + k];
                acc -= ft.AD1[(size_t)a * t.h1 + k] * ft.Phi[(size_t)a * t.D + n];
            }
            acc += dk * X[(size_t)a * t.D + n];
        }
    } else if (p < off_W2(t)) {
        const int m = (p - off_W1(t)) / t.h1, k = (p - off_W1(t)) % t.h1;
        for (int q = lo; q < hi; q++) {
            const int a = satoms[q];
            acc += d1[(size_t)a * t.h2 + m] * H1[(size_t)a * t.h1 + k];
            if (F) acc += ft.fW1[((size_t)a * t.h2 + m) * t.h1 + k];
        }
    } else {
        const int m = p - off_W2(t);
        for (int q = lo; q < hi; q++) {
            const int a = satoms[q];
            acc += ca[a] * H2[(size_t)a * t.h2 + m];
            if (F) acc += ft.fW2[(size_t)a * t.h2 + m];
        }
    }
    grad[idx] = acc / (double)t.S + 2.0 * t.LREG * V[idx];
}

}  // namespace

struct mb_train {
    int device;
    cudaStream_t st;
    TrainDims t;
    int NW;
    double *X, *Eref, *wt, *V, *H1, *H2, *Eat, *Es, *cs, *ls, *d0, *d1, *ca, *grad;
    int *spc, *sat, *soff, *satoms, *soffs;
    double *h_ls;
    long evals;
    /* force training (mb_train_set_forces): NF marked atoms, NB blocks,
     * Nown distinct block owners */
    int NF, NB, Nown;
    double WF;
    int *fatom, *boff, *bown, *bmk, *owners, *ooff, *olist;
    double *Fref, *Fn, *Pj, *AD1, *fpred, *dfq, *lf, *Phi, *Gam, *fB1, *fW1, *fW2, *h_lf;
};

static int tr_cuda(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return MB_OK;
    static __thread char msg[200];
    snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
    return mb_handle_fail(MB_ERR_CUDA, msg);
}

extern "C" int mb_train_close(mb_train *tr) {
    if (!tr) return MB_OK;
    cudaSetDevice(tr->device);
    if (tr->st) cudaStreamSynchronize(tr->st);
    cudaFree(tr->X); cudaFree(tr->Eref); cudaFree(tr->wt); cudaFree(tr->V); cudaFree(tr->grad);
    cudaFree(tr->H1); cudaFree(tr->H2); cudaFree(tr->d0); cudaFree(tr->d1); cudaFree(tr->Eat); cudaFree(tr->ca);
    cudaFree(tr->Es); cudaFree(tr->cs); cudaFree(tr->ls); cudaFree(tr->spc); cudaFree(tr->sat); cudaFree(tr->soff);
    cudaFree(tr->satoms); cudaFree(tr->soffs);
    cudaFree(tr->fatom); cudaFree(tr->boff); cudaFree(tr->bown); cudaFree(tr->bmk); cudaFree(tr->owners);
    cudaFree(tr->ooff); cudaFree(tr->olist); cudaFree(tr->Fref); cudaFree(tr->Fn); cudaFree(tr->Pj);
    cudaFree(tr->AD1); cudaFree(tr->fpred); cudaFree(tr->dfq); cudaFree(tr->lf); cudaFree(tr->Phi);
    cudaFree(tr->Gam); cudaFree(tr->fB1); cudaFree(tr->fW1); cudaFree(tr->fW2);
    cudaFreeHost(tr->h_ls);
    cudaFreeHost(tr->h_lf);
    if (tr->st) cudaStreamDestroy(tr->st);
    free(tr);
    return MB_OK;
}

extern "C" int mb_train_open(int device, int S, const int *nat, const int *atmn, int nspc, int D, int h1, int h2,
                             const double *G, const double *rmin, const double *dr, const double *E_ref,
                             const double *weight, double WE, double LREG, mb_train **out) {
    if (!out || S < 1 || !nat || !atmn || nspc < 1 || nspc > 3 || D < 1 || h1 < 1 || h2 < 1 || h1 > MB_TRAIN_MAXH ||
        h2 > MB_TRAIN_MAXH || !G || !rmin || !dr || !E_ref)
        return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    *out = nullptr;
    int Na = 0;
    for (int s = 0; s < S; s++) {
        if (nat[s] < 1) return mb_handle_fail(MB_ERR_ARG, "empty structure");
        Na += nat[s];
    }
    for (int a = 0; a < Na; a++)
        if (atmn[a] < 0 || atmn[a] >= nspc) return mb_handle_fail(MB_ERR_ARG, "species index out of range");
    mb_train *tr = (mb_train *)calloc(1, sizeof(mb_train));
    tr->device = device;
    tr->t.S = S;
    tr->t.Na = Na;
    tr->t.D = D;
    tr->t.h1 = h1;
    tr->t.h2 = h2;
    tr->t.nspc = nspc;
    tr->t.P = h1 + h2 + 1 + h1 * D + h2 * h1 + h2;
    tr->t.WE = WE;
    tr->t.LREG = LREG;
    tr->NW = nspc * tr->t.P;
    /* host staging: scaled inputs, atom -> structure map, atoms grouped by species */
    double *hX = (double *)malloc(sizeof(double) * (size_t)Na * D);
    int *hsat = (int *)malloc(sizeof(int) * Na), *hsoff = (int *)malloc(sizeof(int) * (S + 1));
    int *hsatoms = (int *)malloc(sizeof(int) * Na), hsoffs[4] = {0, 0, 0, 0};
    double *hw = (double *)malloc(sizeof(double) * S);
    for (int s = 0, a = 0; s < S; s++) {
        hsoff[s] = a;
        hw[s] = weight ? weight[s] : 1.0;
        for (int k = 0; k < nat[s]; k++, a++) hsat[a] = s;
    }
    hsoff[S] = Na;
    for (int a = 0; a < Na; a++) {
        const int sp = atmn[a];
        for (int n = 0; n < D; n++)
            hX[(size_t)a * D + n] = (G[(size_t)a * D + n] - rmin[(size_t)sp * D + n]) * dr[(size_t)sp * D + n];
    }
    {
        int cnt[3] = {0, 0, 0}, k = 0;
        for (int a = 0; a < Na; a++) cnt[atmn[a]]++;
        for (int s = 0; s < nspc; s++) hsoffs[s + 1] = hsoffs[s] + cnt[s];
        for (int s = nspc; s < 3; s++) hsoffs[s + 1] = hsoffs[s];
        for (int s = 0; s < nspc; s++)
            for (int a = 0; a < Na; a++)
                if (atmn[a] == s) hsatoms[k++] = a;
    }
    int rc = tr_cuda(cudaSetDevice(device), "cudaSetDevice");
    if (!rc) rc = tr_cuda(cudaStreamCreateWithFlags(&tr->st, cudaStreamNonBlocking), "cudaStreamCreate");
#define TA(ptr, n) \
    if (!rc) rc = tr_cuda(cudaMalloc((void **)&tr->ptr, sizeof(*tr->ptr) * (size_t)(n)), "cudaMalloc " #ptr)
    TA(X, (size_t)Na * D);
    TA(Eref, S);
    TA(wt, S);
    TA(V, tr->NW);
    TA(grad, tr->NW);
    TA(H1, (size_t)Na * h1);
    TA(H2, (size_t)Na * h2);
    TA(d0, (size_t)Na * h1);
    TA(d1, (size_t)Na * h2);
    TA(Eat, Na);
    TA(ca, Na);
    TA(Es, S);
    TA(cs, S);
    TA(ls, S);
    TA(spc, Na);
    TA(sat, Na);
    TA(soff, S + 1);
    TA(satoms, Na);
    TA(soffs, 4);
#undef TA
    if (!rc) rc = tr_cuda(cudaMemcpy(tr->X, hX, sizeof(double) * (size_t)Na * D, cudaMemcpyHostToDevice), "H2D");
    if (!rc) rc = tr_cuda(cudaMemcpy(tr->Eref, E_ref, sizeof(double) * S, cudaMemcpyHostToDevice), "H2D");
    if (!rc) rc = tr_cuda(cudaMemcpy(tr->wt, hw, sizeof(double) * S, cudaMemcpyHostToDevice), "H2D");
    if (!rc) rc = tr_cuda(cudaMemcpy(tr->spc, atmn, sizeof(int) * Na, cudaMemcpyHostToDevice), "H2D");
    if (!rc) rc = tr_cuda(cudaMemcpy(tr->sat, hsat, sizeof(int) * Na, cudaMemcpyHostToDevice), "H2D");
    if (!rc) rc = tr_cuda(cudaMemcpy(tr->soff, hsoff, sizeof(int) * (S + 1), cudaMemcpyHostToDevice), "H2D");
    if (!rc) rc = tr_cuda(cudaMemcpy(tr->satoms, hsatoms, sizeof(int) * Na, cudaMemcpyHostToDevice), "H2D");
    if (!rc) rc = tr_cuda(cudaMemcpy(tr->soffs, hsoffs, sizeof(int) * 4, cudaMemcpyHostToDevice), "H2D");
    if (!rc) rc = tr_cuda(cudaMallocHost((void **)&tr->h_ls, sizeof(double) * S), "cudaMallocHost");
    free(hX);
    free(hsat);
    free(hsoff);
    free(hsatoms);
    free(hw);
    if (rc) {
        mb_train_close(tr);
        return rc;
    }
    *out = tr;
    return MB_OK;
}

extern "C" int mb_train_info(const mb_train *tr, int *nparams) {
    if (!tr) return mb_handle_fail(MB_ERR_ARG, "null trainer");
    if (nparams) *nparams = tr->NW;
    return MB_OK;
}

extern "C" int mb_train_set_forces(mb_train *tr, int NF, const int *f_atom, const double *F_ref,
                                   const int *blk_off, const int *blk_atom, const double *Fn, int scale_blocks,
                                   const double *dr, double WF) {
    if (!tr || NF < 0 || (NF > 0 && (!f_atom || !F_ref || !blk_off || !blk_atom || !Fn)) || (scale_blocks && !dr))
        return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    const TrainDims &t = tr->t;
    if (tr->NF > 0) return mb_handle_fail(MB_ERR_STATE, "force data already set");
    if (NF == 0) return MB_OK;
    const int NB = blk_off[NF];
    if (blk_off[0] != 0 || NB < NF) return mb_handle_fail(MB_ERR_ARG, "bad block offsets");
    /* atom -> structure, to check that every block belongs to its marked atom's structure */
    int *sat = (int *)malloc(sizeof(int) * t.Na), *atmn = (int *)malloc(sizeof(int) * t.Na);
    int *cnt = (int *)calloc((size_t)t.Na + 1, sizeof(int)), *bmk = (int *)malloc(sizeof(int) * NB);
    int *ooff = nullptr, *olist = nullptr, *owners = nullptr;
    double *hFn = nullptr;
    int rc = MB_OK;
    if (!sat || !atmn || !cnt || !bmk) { rc = mb_handle_fail(MB_ERR_ARG, "out of memory"); goto out; }
    if ((rc = tr_cuda(cudaSetDevice(tr->device), "cudaSetDevice"))) goto out;
    if ((rc = tr_cuda(cudaMemcpy(sat, tr->sat, sizeof(int) * t.Na, cudaMemcpyDeviceToHost), "D2H"))) goto out;
    if ((rc = tr_cuda(cudaMemcpy(atmn, tr->spc, sizeof(int) * t.Na, cudaMemcpyDeviceToHost), "D2H"))) goto out;
    for (int i = 0; i < NF; i++) {
        if (f_atom[i] < 0 || f_atom[i] >= t.Na || blk_off[i + 1] <= blk_off[i]) {
            rc = mb_handle_fail(MB_ERR_ARG, "bad marked atom or empty block list");
            goto out;
        }
        for (int b = blk_off[i]; b < blk_off[i + 1]; b++) {
            const int o = blk_atom[b];
            if (o < 0 || o >= t.Na || sat[o] != sat[f_atom[i]]) {
                rc = mb_handle_fail(MB_ERR_ARG, "block owner outside the marked atom's structure");
                goto out;
            }
            bmk[b] = i;
            cnt[o]++;
        }
    }
    /* blocks grouped by owner atom, in block order */
    ooff = (int *)malloc(sizeof(int) * ((size_t)t.Na + 1));
    olist = (int *)malloc(sizeof(int) * NB);
    owners = (int *)malloc(sizeof(int) * t.Na);
    hFn = (double *)malloc(sizeof(double) * (size_t)NB * t.D * 3);
    if (!ooff || !olist || !owners || !hFn) { rc = mb_handle_fail(MB_ERR_ARG, "out of memory"); goto out; }
    {
        int nown = 0, k = 0;
        int *cur = (int *)malloc(sizeof(int) * t.Na);
        if (!cur) { rc = mb_handle_fail(MB_ERR_ARG, "out of memory"); goto out; }
        for (int a = 0; a < t.Na; a++)
            if (cnt[a]) {
                owners[nown] = a;
                ooff[nown] = k;
                cur[a] = k;
                k += cnt[a];
                nown++;
            }
        ooff[nown] = k;
        for (int b = 0; b < NB; b++) olist[cur[blk_atom[b]]++] = b;
        free(cur);
        tr->Nown = nown;
    }
    /* blocks on the network's input scale: Fn_b[l] DR[s_o][l] (ADJT_LNK, src/nmod.c:244-259) */
    for (int b = 0; b < NB; b++) {
        const int so = atmn[blk_atom[b]];
        for (int l = 0; l < t.D; l++)
            for (int q = 0; q < 3; q++) {
                const size_t k = ((size_t)b * t.D + l) * 3 + q;
                hFn[k] = scale_blocks ? Fn[k] * dr[(size_t)so * t.D + l] : Fn[k];
            }
    }
    tr->NF = NF;
    tr->NB = NB;
    tr->WF = WF;
#define TA(ptr, n) \
    if (!rc) rc = tr_cuda(cudaMalloc((void **)&tr->ptr, sizeof(*tr->ptr) * (size_t)(n)), "cudaMalloc " #ptr)
#define TC(dst, src, n) \
    if (!rc) rc = tr_cuda(cudaMemcpy(tr->dst, src, sizeof(*tr->dst) * (size_t)(n), cudaMemcpyHostToDevice), "H2D " #dst)
    TA(fatom, NF); TA(boff, NF + 1); TA(bown, NB); TA(bmk, NB); TA(owners, tr->Nown); TA(ooff, tr->Nown + 1);
    TA(olist, NB); TA(Fref, 3 * NF); TA(Fn, (size_t)NB * t.D * 3); TA(Pj, (size_t)NB * t.h1 * 3);
    TA(AD1, (size_t)t.Na * t.h1); TA(fpred, 3 * NF); TA(dfq, 3 * NF); TA(lf, NF); TA(Phi, (size_t)t.Na * t.D);
    TA(Gam, (size_t)t.Na * t.h1); TA(fB1, (size_t)t.Na * t.h2); TA(fW1, (size_t)t.Na * t.h2 * t.h1);
    TA(fW2, (size_t)t.Na * t.h2);
    TC(fatom, f_atom, NF); TC(boff, blk_off, NF + 1); TC(bown, blk_atom, NB); TC(bmk, bmk, NB);
    TC(owners, owners, tr->Nown); TC(ooff, ooff, tr->Nown + 1); TC(olist, olist, NB); TC(Fref, F_ref, 3 * NF);
    TC(Fn, hFn, (size_t)NB * t.D * 3);
#undef TA
#undef TC
    /* atoms that own no block keep zero force terms */
    if (!rc) rc = tr_cuda(cudaMemset(tr->Phi, 0, sizeof(double) * (size_t)t.Na * t.D), "memset");
    if (!rc) rc = tr_cuda(cudaMemset(tr->Gam, 0, sizeof(double) * (size_t)t.Na * t.h1), "memset");
    if (!rc) rc = tr_cuda(cudaMemset(tr->fB1, 0, sizeof(double) * (size_t)t.Na * t.h2), "memset");
    if (!rc) rc = tr_cuda(cudaMemset(tr->fW1, 0, sizeof(double) * (size_t)t.Na * t.h2 * t.h1), "memset");
    if (!rc) rc = tr_cuda(cudaMemset(tr->fW2, 0, sizeof(double) * (size_t)t.Na * t.h2), "memset");
    if (!rc) rc = tr_cuda(cudaMallocHost((void **)&tr->h_lf, sizeof(double) * NF), "cudaMallocHost");
out:
    free(sat); free(atmn); free(cnt); free(bmk); free(ooff); free(olist); free(owners); free(hFn);
    return rc;
}

/* forward pass, forces and (with grad) the gradient; the loss terms land in h_ls / h_lf */
static int tr_run(mb_train *tr, const double *V, double *grad) {
    const TrainDims &t = tr->t;
    cudaStream_t st = tr->st;
    int rc = tr_cuda(cudaSetDevice(tr->device), "cudaSetDevice");
    if (!rc) rc = tr_cuda(cudaMemcpyAsync(tr->V, V, sizeof(double) * tr->NW, cudaMemcpyHostToDevice, st), "H2D V");
    if (rc) return rc;
    const bool F = tr->NF > 0;
    k_tr_fwd<<<(t.Na + 3) / 4, 128, 0, st>>>(t, tr->X, tr->spc, tr->V, tr->H1, tr->H2, tr->Eat);
    k_tr_struct<<<(t.S + 127) / 128, 128, 0, st>>>(t, tr->soff, tr->Eat, tr->Eref, tr->wt, tr->Es, tr->cs, tr->ls);
    if (F) {
        k_tr_ad1<<<(t.Na + 127) / 128, 128, 0, st>>>(t, tr->spc, tr->V, tr->H1, tr->H2, tr->AD1);
        k_tr_fproj<<<tr->NB, 128, 0, st>>>(t, tr->NB, tr->bown, tr->spc, tr->V, tr->Fn, tr->Pj);
        k_tr_frc<<<(tr->NF + 3) / 4, 128, 0, st>>>(t, tr->NF, tr->fatom, tr->boff, tr->bown, tr->sat, tr->wt,
                                                   tr->Fref, tr->AD1, tr->Pj, tr->WF, tr->fpred, tr->dfq, tr->lf);
    }
    if (grad) {
        k_tr_delta<<<(t.Na + 127) / 128, 128, 0, st>>>(t, tr->spc, tr->sat, tr->V, tr->H1, tr->H2, tr->cs, tr->d0,
                                                       tr->d1, tr->ca);
        ForceTerms ft = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
        if (F) {
            k_tr_fown<<<tr->Nown, 128, sizeof(double) * t.D, st>>>(t, tr->owners, tr->ooff, tr->olist, tr->bmk,
                                                                   tr->spc, tr->V, tr->H1, tr->H2, tr->Fn, tr->Pj,
                                                                   tr->dfq, tr->Phi, tr->Gam, tr->fB1, tr->fW1,
                                                                   tr->fW2);
            ft = {tr->AD1, tr->Phi, tr->Gam, tr->fB1, tr->fW1, tr->fW2};
        }
        k_tr_grad<<<(tr->NW + 127) / 128, 128, 0, st>>>(t, tr->satoms, tr->soffs, tr->X, tr->H1, tr->H2, tr->d0,
                                                        tr->d1, tr->ca, ft, tr->V, tr->grad);
    }
    rc = tr_cuda(cudaGetLastError(), "training kernels");
    if (!rc) rc = tr_cuda(cudaMemcpyAsync(tr->h_ls, tr->ls, sizeof(double) * t.S, cudaMemcpyDeviceToHost, st), "D2H");
    if (!rc && F)
        rc = tr_cuda(cudaMemcpyAsync(tr->h_lf, tr->lf, sizeof(double) * tr->NF, cudaMemcpyDeviceToHost, st), "D2H");
    if (!rc && grad)
        rc = tr_cuda(cudaMemcpyAsync(grad, tr->grad, sizeof(double) * tr->NW, cudaMemcpyDeviceToHost, st), "D2H");
    return rc;
}

extern "C" int mb_train_eval(mb_train *tr, const double *V, double *RT, double *grad, double *E_pred) {
    if (!tr || !V || !RT) return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    const TrainDims &t = tr->t;
    int rc = tr_run(tr, V, grad);
    if (!rc && E_pred)
        rc = tr_cuda(cudaMemcpyAsync(E_pred, tr->Es, sizeof(double) * t.S, cudaMemcpyDeviceToHost, tr->st), "D2H");
    if (!rc) rc = tr_cuda(cudaStreamSynchronize(tr->st), "synchronize");
    if (rc) return rc;
    /* the objective of tot_err_gsl (src/nmin.c:111-166), summed in order */
    double re = 0.0, rf = 0.0, reg = 0.0;
    for (int s = 0; s < t.S; s++) re += tr->h_ls[s];
    for (int i = 0; i < tr->NF; i++) rf += tr->h_lf[i];
    for (int k = 0; k < tr->NW; k++) reg += V[k] * V[k];
    *RT = (re * t.WE + rf * tr->WF) / (double)t.S + t.LREG * reg;
    tr->evals++;
    return MB_OK;
}

extern "C" int mb_train_eval_forces(mb_train *tr, const double *V, double *f_pred, double *RF) {
    if (!tr || !V) return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    if (tr->NF == 0) return mb_handle_fail(MB_ERR_STATE, "no force data");
    int rc = tr_run(tr, V, nullptr);
    if (!rc && f_pred)
        rc = tr_cuda(cudaMemcpyAsync(f_pred, tr->fpred, sizeof(double) * 3 * tr->NF, cudaMemcpyDeviceToHost, tr->st),
                     "D2H");
    if (!rc) rc = tr_cuda(cudaStreamSynchronize(tr->st), "synchronize");
    if (rc) return rc;
    if (RF) {
        double rf = 0.0;
        for (int i = 0; i < tr->NF; i++) rf += tr->h_lf[i];
        *RF = rf;
    }
    return MB_OK;
}

typedef struct {
    mb_train *tr;
    int err;
} fit_ctx;

static double fit_f(void *c, double *x) {
    fit_ctx *f = (fit_ctx *)c;
    double RT = NAN;
    if (!f->err) f->err = mb_train_eval(f->tr, x, &RT, nullptr, nullptr);
    return f->err ? NAN : RT;
}

static double fit_fg(void *c, double *x, double *g) {
    fit_ctx *f = (fit_ctx *)c;
    double RT = NAN;
    if (!f->err) f->err = mb_train_eval(f->tr, x, &RT, g, nullptr);
    return f->err ? NAN : RT;
}

extern "C" int mb_train_fit(mb_train *tr, double *V, int mitr, double gtol, double *RT, int *iters) {
    if (!tr || !V || mitr < 0) return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    fit_ctx c = {tr, 0};
    mb_bfgs b;
    /* MLP_MIN's minimiser set-up: initial step 0.01, line tolerance 1e-5 (src/nmin.c:389-390) */
    if (mb_bfgs_init(&b, tr->NW, V, 0.01, 1e-5, fit_f, fit_fg, &c)) return mb_handle_fail(MB_ERR_ARG, "out of memory");
    int it = 0;
    while (!c.err && it < mitr) {
        double gg = 0.0;
        for (int k = 0; k < tr->NW; k++) gg += b.g[k] * b.g[k];
        if (sqrt(gg) < gtol) break; /* gsl_multimin_test_gradient (src/nmin.c:411) */
        it++;
        if (mb_bfgs_iterate(&b) != MB_BFGS_OK && !c.err) {
            /* no acceptable step: restart from steepest descent once, as
             * MLP_MIN restarts its minimiser (src/nmin.c:396-403) */
            mb_bfgs_restart(&b);
            if (mb_bfgs_iterate(&b) != MB_BFGS_OK) break;
        }
    }
    const int rc = c.err;
    if (!rc) {
        memcpy(V, b.x, sizeof(double) * tr->NW);
        if (RT) *RT = b.f;
        if (iters) *iters = it;
    }
    mb_bfgs_free(&b);
    return rc;
}
