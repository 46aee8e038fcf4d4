/*
 * mb_train.cu -- training of the per-species MLP on the GPU: the objective
 * and gradient of MAISE's network training (tot_err_gsl / dfunc_gsl,
 * src/nmin.c:93-305, with the energy back-propagation of DE_ANN_PARA,
 * src/nmlp.c:292-354), minimised by the project BFGS (mb_bfgs.c) as
 * MLP_MIN does with GSL's vector_bfgs2 (src/nmin.c:314-445).
 *
 * Objective over S training structures with reference energies E_s,
 * weights w_s and atoms N_s:
 *   RT = WE sum_s w_s ((E_s - E(s)) / N_s)^2 / S + LREG sum(b^2 + W^2),
 *   E(s) = sum over the structure's atoms of the species network on the
 *   scaled inputs x = (G - Rmin) DR,
 * and its gradient: the back-propagated c_s = 2 WE w_s (E(s) - E_s) / N_s^2
 * summed over atoms, / S, plus 2 LREG V.  The reference's force term
 * (DF_ANN_PARA, src/nmlp.c:104-130) adds nothing to the gradient, so the
 * trainer works with energies, as the reference does.
 *
 * Parameters in the reference's V2W order (src/nmlp.c:591-608): per species
 * the biases of all layers (b0[h1], b1[h2], b2), then the weights
 * W0[h1][D], W1[h2][h1], W2[h2].  Hidden layers tanh, output linear.
 *
 * Kernels (FP64; every sum in a fixed order, so results are reproducible):
 *   k_tr_fwd     one warp per atom: hidden activations and the atom energy
 *   k_tr_struct  one thread per structure: E(s), c_s and the loss term
 *   k_tr_delta   one thread per atom: back-propagated deltas
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

/* one thread per parameter of one species: the sum over that species'
 * atoms (in atom order) of the parameter's back-propagated term */
__global__ void k_tr_grad(TrainDims t, const int *__restrict__ satoms, const int *__restrict__ soffs,
                          const double *__restrict__ X, const double *__restrict__ H1, const double *__restrict__ H2,
                          const double *__restrict__ d0, const double *__restrict__ d1, const double *__restrict__ ca,
                          const double *__restrict__ V, double *__restrict__ grad) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= t.nspc * t.P) return;
    const int s = idx / t.P, p = idx % t.P;
    const int lo = soffs[s], hi = soffs[s + 1];
    double acc = 0.0;
    if (p < off_b1(t)) {
        const int k = p;
        for (int q = lo; q < hi; q++) acc += d0[(size_t)satoms[q] * t.h1 + k];
    } else if (p < off_b2(t)) {
        const int m = p - off_b1(t);
        for (int q = lo; q < hi; q++) acc += d1[(size_t)satoms[q] * t.h2 + m];
    } else if (p < off_W0(t)) {
        for (int q = lo; q < hi; q++) acc += ca[satoms[q]];
    } else if (p < off_W1(t)) {
        const int k = (p - off_W0(t)) / t.D, n = (p - off_W0(t)) % t.D;
        for (int q = lo; q < hi; q++) {
            const int a = satoms[q];
            acc += d0[(size_t)a * t.h1 + k] * X[(size_t)a * t.D + n];
        }
    } else if (p < off_W2(t)) {
        const int m = (p - off_W1(t)) / t.h1, k = (p - off_W1(t)) % t.h1;
        for (int q = lo; q < hi; q++) {
            const int a = satoms[q];
            acc += d1[(size_t)a * t.h2 + m] * H1[(size_t)a * t.h1 + k];
        }
    } else {
        const int m = p - off_W2(t);
        for (int q = lo; q < hi; q++) {
            const int a = satoms[q];
            acc += ca[a] * H2[(size_t)a * t.h2 + m];
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
    cudaFreeHost(tr->h_ls);
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

extern "C" int mb_train_eval(mb_train *tr, const double *V, double *RT, double *grad, double *E_pred) {
    if (!tr || !V || !RT) return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    const TrainDims &t = tr->t;
    cudaStream_t st = tr->st;
    int rc = tr_cuda(cudaSetDevice(tr->device), "cudaSetDevice");
    if (!rc) rc = tr_cuda(cudaMemcpyAsync(tr->V, V, sizeof(double) * tr->NW, cudaMemcpyHostToDevice, st), "H2D V");
    if (rc) return rc;
    k_tr_fwd<<<(t.Na + 3) / 4, 128, 0, st>>>(t, tr->X, tr->spc, tr->V, tr->H1, tr->H2, tr->Eat);
    k_tr_struct<<<(t.S + 127) / 128, 128, 0, st>>>(t, tr->soff, tr->Eat, tr->Eref, tr->wt, tr->Es, tr->cs, tr->ls);
    if (grad) {
        k_tr_delta<<<(t.Na + 127) / 128, 128, 0, st>>>(t, tr->spc, tr->sat, tr->V, tr->H1, tr->H2, tr->cs, tr->d0,
                                                       tr->d1, tr->ca);
        k_tr_grad<<<(tr->NW + 127) / 128, 128, 0, st>>>(t, tr->satoms, tr->soffs, tr->X, tr->H1, tr->H2, tr->d0,
                                                        tr->d1, tr->ca, tr->V, tr->grad);
    }
    rc = tr_cuda(cudaGetLastError(), "training kernels");
    if (!rc) rc = tr_cuda(cudaMemcpyAsync(tr->h_ls, tr->ls, sizeof(double) * t.S, cudaMemcpyDeviceToHost, st), "D2H");
    if (!rc && grad)
        rc = tr_cuda(cudaMemcpyAsync(grad, tr->grad, sizeof(double) * tr->NW, cudaMemcpyDeviceToHost, st), "D2H");
    if (!rc && E_pred)
        rc = tr_cuda(cudaMemcpyAsync(E_pred, tr->Es, sizeof(double) * t.S, cudaMemcpyDeviceToHost, st), "D2H");
    if (!rc) rc = tr_cuda(cudaStreamSynchronize(st), "synchronize");
    if (rc) return rc;
    /* the objective of tot_err_gsl (src/nmin.c:150-166), summed in order */
    double re = 0.0, reg = 0.0;
    for (int s = 0; s < t.S; s++) re += tr->h_ls[s];
    for (int k = 0; k < tr->NW; k++) reg += V[k] * V[k];
    *RT = re * t.WE / (double)t.S + t.LREG * reg;
    tr->evals++;
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
