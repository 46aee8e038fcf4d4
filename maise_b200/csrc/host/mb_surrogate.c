/*
 * mb_surrogate.c -- host side of the surrogate screen (include/maise_surrogate.h):
 * network state on the GPU, the training loop, prediction and the check
 * entry points.  The kernels are in cuda/mb_surrogate.cu.
 */
#include <cuda_runtime_api.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../../../include/maise_surrogate.h"
#include "mb_surrogate_k.h"

int mb_handle_fail(int code, const char *msg);

#define NL 4 /* dense layers */

struct mb_surrogate {
    int device;
    cudaStream_t st;
    int nspc, nbins, nin;
    double rmax, sigma;
    int dims[NL + 1];
    long np, woff[NL], boff[NL];
    float *p, *g, *m, *v;   /* parameters, gradient, Adam moments */
    float *mean, *istd;     /* feature standardisation */
    double tmean, tstd;     /* target standardisation */
    long t;                 /* Adam steps taken */
    int bcap;               /* rows the work buffers hold */
    float *x, *tt, *z[NL], *a[NL], *dz[NL];
    int *idx;
    double *loss;
    int loss_cap;
};

#define CK(call)                                                                   \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) return mb_handle_fail(MB_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)
#define KK(call)                                                                   \
    do {                                                                           \
        int e_ = (call);                                                           \
        if (e_) return mb_handle_fail(MB_ERR_CUDA, cudaGetErrorString((cudaError_t)e_)); \
    } while (0)

/* splitmix64: seeds the weight initialisation and the epoch shuffles */
static uint64_t sm_next(uint64_t *s) {
    uint64_t z = (*s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static double sm_unif(uint64_t *s) { return ((sm_next(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
static double sm_normal(uint64_t *s) { /* Box-Muller */
    const double u = sm_unif(s), w = sm_unif(s);
    return sqrt(-2.0 * log(u)) * cos(2.0 * M_PI * w);
}

static void free_work(mb_surrogate *s) {
    int l;
    cudaFree(s->x);
    cudaFree(s->tt);
    cudaFree(s->idx);
    for (l = 0; l < NL; l++) {
        cudaFree(s->z[l]);
        cudaFree(s->a[l]);
        cudaFree(s->dz[l]);
        s->z[l] = s->a[l] = s->dz[l] = NULL;
    }
    s->x = s->tt = NULL;
    s->idx = NULL;
    s->bcap = 0;
}

/* work buffers for B rows */
static int ensure_rows(mb_surrogate *s, int B) {
    int l;
    if (B <= s->bcap) return MB_OK;
    free_work(s);
    CK(cudaMalloc((void **)&s->x, sizeof(float) * (size_t)B * s->nin));
    CK(cudaMalloc((void **)&s->tt, sizeof(float) * B));
    CK(cudaMalloc((void **)&s->idx, sizeof(int) * B));
    for (l = 0; l < NL; l++) {
        const size_t n = (size_t)B * s->dims[l + 1];
        CK(cudaMalloc((void **)&s->z[l], sizeof(float) * n));
        CK(cudaMalloc((void **)&s->a[l], sizeof(float) * n));
        CK(cudaMalloc((void **)&s->dz[l], sizeof(float) * n));
    }
    s->bcap = B;
    return MB_OK;
}

static int ensure_loss(mb_surrogate *s, int n) {
    if (n <= s->loss_cap) return MB_OK;
    cudaFree(s->loss);
    s->loss = NULL;
    CK(cudaMalloc((void **)&s->loss, sizeof(double) * n));
    s->loss_cap = n;
    return MB_OK;
}

static int init_state(mb_surrogate *s, unsigned seed);

int mb_sur_open(int device, int nspc, int nbins, double rmax, double sigma, int h1, int h2, int h3, unsigned seed,
                mb_surrogate **out) {
    mb_surrogate *s;
    long o = 0;
    int l, ndev = 0;
    if (!out || nspc < 1 || nspc > SUR_MAX_SPC || nbins < 1 || !(rmax > 0) || !(sigma > 0) || h1 < 1 || h2 < 1 ||
        h3 < 1)
        return mb_handle_fail(MB_ERR_ARG, "bad surrogate shape");
    if ((size_t)nbins * nspc * (nspc + 1) / 2 * sizeof(float) > 48 * 1024)
        return mb_handle_fail(MB_ERR_ARG, "histogram too large for one CTA's shared memory");
    *out = NULL;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return mb_handle_fail(MB_ERR_NOGPU, "no CUDA device");
    if (device < 0 || device >= ndev) return mb_handle_fail(MB_ERR_ARG, "device out of range");
    CK(cudaSetDevice(device));
    s = (mb_surrogate *)calloc(1, sizeof(*s));
    s->device = device;
    s->nspc = nspc;
    s->nbins = nbins;
    s->rmax = rmax;
    s->sigma = sigma;
    s->nin = nbins * nspc * (nspc + 1) / 2;
    s->dims[0] = s->nin;
    s->dims[1] = h1;
    s->dims[2] = h2;
    s->dims[3] = h3;
    s->dims[4] = 1;
    for (l = 0; l < NL; l++) {
        s->woff[l] = o;
        o += (long)s->dims[l + 1] * s->dims[l];
        s->boff[l] = o;
        o += s->dims[l + 1];
    }
    s->np = o;
    s->tstd = 1.0;
    if ((l = init_state(s, seed))) {
        mb_sur_close(s);
        return l;
    }
    *out = s;
    return MB_OK;
}

static int init_state(mb_surrogate *s, unsigned seed) {
    float *hp;
    uint64_t rs = seed;
    int l;
    CK(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
    CK(cudaMalloc((void **)&s->p, sizeof(float) * s->np));
    CK(cudaMalloc((void **)&s->g, sizeof(float) * s->np));
    CK(cudaMalloc((void **)&s->m, sizeof(float) * s->np));
    CK(cudaMalloc((void **)&s->v, sizeof(float) * s->np));
    CK(cudaMalloc((void **)&s->mean, sizeof(float) * s->nin));
    CK(cudaMalloc((void **)&s->istd, sizeof(float) * s->nin));
    CK(cudaMemset(s->m, 0, sizeof(float) * s->np));
    CK(cudaMemset(s->v, 0, sizeof(float) * s->np));
    CK(cudaMemset(s->mean, 0, sizeof(float) * s->nin));
    hp = (float *)malloc(sizeof(float) * (s->np > s->nin ? s->np : s->nin));
    for (l = 0; l < NL; l++) {
        const long nw = (long)s->dims[l + 1] * s->dims[l];
        const double sd = 1.0 / sqrt((double)s->dims[l]);
        long k;
        for (k = 0; k < nw; k++) hp[s->woff[l] + k] = (float)(sd * sm_normal(&rs));
        for (k = 0; k < s->dims[l + 1]; k++) hp[s->boff[l] + k] = 0.0f;
    }
    if (cudaMemcpy(s->p, hp, sizeof(float) * s->np, cudaMemcpyHostToDevice) != cudaSuccess) {
        free(hp);
        return mb_handle_fail(MB_ERR_CUDA, "parameter upload");
    }
    for (l = 0; l < s->nin; l++) hp[l] = 1.0f;
    if (cudaMemcpy(s->istd, hp, sizeof(float) * s->nin, cudaMemcpyHostToDevice) != cudaSuccess) {
        free(hp);
        return mb_handle_fail(MB_ERR_CUDA, "standardisation upload");
    }
    free(hp);
    return MB_OK;
}

void mb_sur_close(mb_surrogate *s) {
    if (!s) return;
    cudaSetDevice(s->device);
    free_work(s);
    cudaFree(s->p);
    cudaFree(s->g);
    cudaFree(s->m);
    cudaFree(s->v);
    cudaFree(s->mean);
    cudaFree(s->istd);
    cudaFree(s->loss);
    if (s->st) cudaStreamDestroy(s->st);
    free(s);
}

int mb_sur_info(const mb_surrogate *s, int *nin, long *nparams) {
    if (!s) return mb_handle_fail(MB_ERR_ARG, "null handle");
    if (nin) *nin = s->nin;
    if (nparams) *nparams = s->np;
    return MB_OK;
}

/* ------------------------------------------------------------- network */

/* forward pass over B standardised rows at x; the output lands in z[NL-1] */
static int forward(mb_surrogate *s, int B, const float *x) {
    const float *in = x;
    int l;
    for (l = 0; l < NL; l++) {
        const int I = s->dims[l], O = s->dims[l + 1];
        const float *W = s->p + s->woff[l], *b = s->p + s->boff[l];
        if (l < NL - 1) {
            KK(surk_gemm(0, 1, SUR_EP_BIAS_SILU, B, O, I, in, I, W, I, s->a[l], O, b, s->z[l], NULL, s->st));
            in = s->a[l];
        } else {
            KK(surk_gemm(0, 1, SUR_EP_BIAS, B, O, I, in, I, W, I, s->z[l], O, b, NULL, NULL, s->st));
        }
    }
    return MB_OK;
}

/* loss into *dloss and the gradient into s->g, after forward() on the same rows */
static int backward(mb_surrogate *s, int B, const float *x, const float *t, double *dloss) {
    int l;
    KK(surk_mse(B, s->z[NL - 1], t, s->dz[NL - 1], dloss, s->st));
    for (l = NL - 1; l >= 0; l--) {
        const int I = s->dims[l], O = s->dims[l + 1];
        const float *in = l ? s->a[l - 1] : x;
        KK(surk_gemm(1, 0, SUR_EP_STORE, O, I, B, s->dz[l], O, in, I, s->g + s->woff[l], I, NULL, NULL, NULL, s->st));
        KK(surk_colsum(B, O, s->dz[l], s->g + s->boff[l], s->st));
        if (l)
            KK(surk_gemm(0, 0, SUR_EP_DSILU, B, I, O, s->dz[l], O, s->p + s->woff[l], I, s->dz[l - 1], I, NULL, NULL,
                         s->z[l - 1], s->st));
    }
    return MB_OK;
}

static int adam(mb_surrogate *s, double lr) {
    const double b1 = 0.9, b2 = 0.999;
    s->t++;
    KK(surk_adam(s->np, s->p, s->g, s->m, s->v, (float)lr, (float)b1, (float)b2, 1e-8f,
                 (float)(1.0 / (1.0 - pow(b1, (double)s->t))), (float)(1.0 / (1.0 - pow(b2, (double)s->t))), s->st));
    return MB_OK;
}

/* ------------------------------------------------------------ features */

typedef struct {
    int *off, *spc;
    double *lat, *x;
    int *status;
    int total;
} dev_structs;

static void free_structs(dev_structs *d) {
    cudaFree(d->off);
    cudaFree(d->spc);
    cudaFree(d->lat);
    cudaFree(d->x);
    cudaFree(d->status);
    memset(d, 0, sizeof(*d));
}

static int upload_structs(mb_surrogate *s, int S, const int *nat, const int *atmn, const double *lat, const double *x,
                          dev_structs *d) {
    int *off, k, total = 0;
    cudaError_t e;
    memset(d, 0, sizeof(*d));
    off = (int *)malloc(sizeof(int) * (S + 1));
    for (k = 0; k < S; k++) {
        if (nat[k] < 1 || nat[k] > SUR_MAX_ATOMS) {
            free(off);
            return mb_handle_fail(MB_ERR_ARG, "the surrogate takes 1..256 atoms per structure");
        }
        off[k] = total;
        total += nat[k];
    }
    off[S] = total;
    for (k = 0; k < total; k++)
        if (atmn[k] < 0 || atmn[k] >= s->nspc) {
            free(off);
            return mb_handle_fail(MB_ERR_ARG, "species index out of range");
        }
    d->total = total;
    e = cudaMalloc((void **)&d->off, sizeof(int) * (S + 1));
    if (!e) e = cudaMalloc((void **)&d->spc, sizeof(int) * total);
    if (!e) e = cudaMalloc((void **)&d->lat, sizeof(double) * 9 * S);
    if (!e) e = cudaMalloc((void **)&d->x, sizeof(double) * 3 * total);
    if (!e) e = cudaMalloc((void **)&d->status, sizeof(int));
    if (!e) e = cudaMemcpyAsync(d->off, off, sizeof(int) * (S + 1), cudaMemcpyHostToDevice, s->st);
    if (!e) e = cudaMemcpyAsync(d->spc, atmn, sizeof(int) * total, cudaMemcpyHostToDevice, s->st);
    if (!e) e = cudaMemcpyAsync(d->lat, lat, sizeof(double) * 9 * S, cudaMemcpyHostToDevice, s->st);
    if (!e) e = cudaMemcpyAsync(d->x, x, sizeof(double) * 3 * total, cudaMemcpyHostToDevice, s->st);
    if (!e) e = cudaMemsetAsync(d->status, 0, sizeof(int), s->st);
    if (!e) e = cudaStreamSynchronize(s->st); /* `off` is pageable and freed next */
    free(off);
    if (e) {
        free_structs(d);
        return mb_handle_fail(MB_ERR_CUDA, cudaGetErrorString(e));
    }
    return MB_OK;
}

static int run_rdf(mb_surrogate *s, int S, dev_structs *d, float *d_feat) {
    int status = 0;
    KK(surk_rdf(S, d->off, d->spc, d->lat, d->x, s->nspc, s->nbins, s->rmax, s->sigma, d_feat, d->status, s->st));
    CK(cudaMemcpyAsync(&status, d->status, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (status)
        return mb_handle_fail(MB_ERR_ARG, "a cell is degenerate or too thin for the histogram range (more than 6 "
                                          "periodic images per direction)");
    return MB_OK;
}

int mb_sur_features(mb_surrogate *s, int S, const int *nat, const int *atmn, const double *lat, const double *x,
                    float *feat) {
    dev_structs d;
    float *d_feat = NULL;
    int rc;
    if (!s || S < 1 || !nat || !atmn || !lat || !x || !feat) return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    CK(cudaSetDevice(s->device));
    if ((rc = upload_structs(s, S, nat, atmn, lat, x, &d))) return rc;
    if (cudaMalloc((void **)&d_feat, sizeof(float) * (size_t)S * s->nin) != cudaSuccess) {
        free_structs(&d);
        return mb_handle_fail(MB_ERR_CUDA, "cudaMalloc features");
    }
    rc = run_rdf(s, S, &d, d_feat);
    if (!rc && cudaMemcpy(feat, d_feat, sizeof(float) * (size_t)S * s->nin, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = mb_handle_fail(MB_ERR_CUDA, "feature download");
    cudaFree(d_feat);
    free_structs(&d);
    return rc;
}

/* ---------------------------------------------------------- prediction */

#define PRED_CHUNK 4096

static int predict_dev(mb_surrogate *s, int S, const float *d_feat, double *pred) {
    float *y;
    int c0, k, rc;
    if ((rc = ensure_rows(s, PRED_CHUNK))) return rc;
    y = (float *)malloc(sizeof(float) * PRED_CHUNK);
    for (c0 = 0; c0 < S; c0 += PRED_CHUNK) {
        const int B = S - c0 < PRED_CHUNK ? S - c0 : PRED_CHUNK;
        int e = surk_gather(B, s->nin, NULL, d_feat + (size_t)c0 * s->nin, s->mean, s->istd, s->x, NULL, 0.0f, 1.0f,
                            NULL, s->st);
        if (e) {
            free(y);
            return mb_handle_fail(MB_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
        }
        if ((rc = forward(s, B, s->x))) {
            free(y);
            return rc;
        }
        if (cudaMemcpyAsync(y, s->z[NL - 1], sizeof(float) * B, cudaMemcpyDeviceToHost, s->st) != cudaSuccess ||
            cudaStreamSynchronize(s->st) != cudaSuccess) {
            free(y);
            return mb_handle_fail(MB_ERR_CUDA, "prediction download");
        }
        for (k = 0; k < B; k++) pred[c0 + k] = (double)y[k] * s->tstd + s->tmean;
    }
    free(y);
    return MB_OK;
}

int mb_sur_predict(mb_surrogate *s, int S, const float *feat, double *pred) {
    float *d_feat = NULL;
    int rc;
    if (!s || S < 1 || !feat || !pred) return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    CK(cudaSetDevice(s->device));
    CK(cudaMalloc((void **)&d_feat, sizeof(float) * (size_t)S * s->nin));
    if (cudaMemcpyAsync(d_feat, feat, sizeof(float) * (size_t)S * s->nin, cudaMemcpyHostToDevice, s->st) !=
        cudaSuccess) {
        cudaFree(d_feat);
        return mb_handle_fail(MB_ERR_CUDA, "feature upload");
    }
    rc = predict_dev(s, S, d_feat, pred);
    cudaFree(d_feat);
    return rc;
}

int mb_sur_screen(mb_surrogate *s, int S, const int *nat, const int *atmn, const double *lat, const double *x,
                  double *pred) {
    dev_structs d;
    float *d_feat = NULL;
    int rc;
    if (!s || S < 1 || !nat || !atmn || !lat || !x || !pred) return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    CK(cudaSetDevice(s->device));
    if ((rc = upload_structs(s, S, nat, atmn, lat, x, &d))) return rc;
    if (cudaMalloc((void **)&d_feat, sizeof(float) * (size_t)S * s->nin) != cudaSuccess) {
        free_structs(&d);
        return mb_handle_fail(MB_ERR_CUDA, "cudaMalloc features");
    }
    rc = run_rdf(s, S, &d, d_feat);
    if (!rc) rc = predict_dev(s, S, d_feat, pred);
    cudaFree(d_feat);
    free_structs(&d);
    return rc;
}

/* ------------------------------------------------------------ training */

int mb_sur_fit(mb_surrogate *s, int S, const float *feat, const double *y, int epochs, int batch, double lr,
               unsigned seed, float *loss) {
    float *d_feat = NULL, *d_y = NULL, *hy;
    int *perm, *d_perm = NULL, ep, k, rc = MB_OK;
    double mu = 0.0, var = 0.0, *hl = NULL;
    uint64_t rs = seed;
    const int nb = (S + batch - 1) / (batch > 0 ? batch : 1);
    if (!s || S < 2 || !feat || !y || epochs < 0 || batch < 1 || !(lr > 0))
        return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    CK(cudaSetDevice(s->device));
    if ((rc = ensure_rows(s, batch)) || (rc = ensure_loss(s, nb))) return rc;
    for (k = 0; k < S; k++) mu += y[k];
    mu /= S;
    for (k = 0; k < S; k++) var += (y[k] - mu) * (y[k] - mu);
    s->tmean = mu;
    s->tstd = sqrt(var / S) > 1e-12 ? sqrt(var / S) : 1.0;
    hy = (float *)malloc(sizeof(float) * S);
    perm = (int *)malloc(sizeof(int) * S);
    hl = (double *)malloc(sizeof(double) * nb);
    for (k = 0; k < S; k++) hy[k] = (float)y[k];
    {
        cudaError_t e = cudaMalloc((void **)&d_feat, sizeof(float) * (size_t)S * s->nin);
        if (!e) e = cudaMalloc((void **)&d_y, sizeof(float) * S);
        if (!e) e = cudaMalloc((void **)&d_perm, sizeof(int) * S);
        if (!e) e = cudaMemcpyAsync(d_feat, feat, sizeof(float) * (size_t)S * s->nin, cudaMemcpyHostToDevice, s->st);
        if (!e) e = cudaMemcpyAsync(d_y, hy, sizeof(float) * S, cudaMemcpyHostToDevice, s->st);
        if (!e) e = (cudaError_t)surk_colstats(S, s->nin, d_feat, s->mean, s->istd, s->st);
        if (!e) e = cudaStreamSynchronize(s->st);
        if (e) {
            rc = mb_handle_fail(MB_ERR_CUDA, cudaGetErrorString(e));
            goto out;
        }
    }
    for (ep = 0; ep < epochs; ep++) {
        double sum = 0.0;
        int b;
        for (k = 0; k < S; k++) perm[k] = k;
        for (k = S - 1; k > 0; k--) { /* Fisher-Yates */
            const int j = (int)(sm_next(&rs) % (uint64_t)(k + 1));
            const int t = perm[k];
            perm[k] = perm[j];
            perm[j] = t;
        }
        if (cudaMemcpyAsync(d_perm, perm, sizeof(int) * S, cudaMemcpyHostToDevice, s->st) != cudaSuccess) {
            rc = mb_handle_fail(MB_ERR_CUDA, "permutation upload");
            goto out;
        }
        for (b = 0; b < nb; b++) {
            const int r0 = b * batch, B = S - r0 < batch ? S - r0 : batch;
            const float tistd = (float)(1.0 / s->tstd);
            int e = surk_gather(B, s->nin, d_perm + r0, d_feat, s->mean, s->istd, s->x, d_y, (float)s->tmean, tistd,
                                s->tt, s->st);
            if (e) {
                rc = mb_handle_fail(MB_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
                goto out;
            }
            if ((rc = forward(s, B, s->x)) || (rc = backward(s, B, s->x, s->tt, s->loss + b)) || (rc = adam(s, lr)))
                goto out;
        }
        /* the permutation buffer is rewritten next epoch: wait for this one */
        if (cudaMemcpyAsync(hl, s->loss, sizeof(double) * nb, cudaMemcpyDeviceToHost, s->st) != cudaSuccess ||
            cudaStreamSynchronize(s->st) != cudaSuccess) {
            rc = mb_handle_fail(MB_ERR_CUDA, "training step failed");
            goto out;
        }
        for (b = 0; b < nb; b++) sum += hl[b];
        if (loss) loss[ep] = (float)(sum / nb);
    }
out:
    cudaStreamSynchronize(s->st);
    cudaFree(d_feat);
    cudaFree(d_y);
    cudaFree(d_perm);
    free(hy);
    free(perm);
    free(hl);
    return rc;
}

/* --------------------------------------------------------------- checks */

int mb_sur_loss_grad(mb_surrogate *s, int B, const float *x, const float *t, double *loss, float *grad) {
    int rc;
    if (!s || B < 1 || !x || !t || !loss || !grad) return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    CK(cudaSetDevice(s->device));
    if ((rc = ensure_rows(s, B)) || (rc = ensure_loss(s, 1))) return rc;
    CK(cudaMemcpyAsync(s->x, x, sizeof(float) * (size_t)B * s->nin, cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->tt, t, sizeof(float) * B, cudaMemcpyHostToDevice, s->st));
    if ((rc = forward(s, B, s->x)) || (rc = backward(s, B, s->x, s->tt, s->loss))) return rc;
    CK(cudaMemcpyAsync(loss, s->loss, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaMemcpyAsync(grad, s->g, sizeof(float) * s->np, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return MB_OK;
}

int mb_sur_adam_step(mb_surrogate *s, const float *grad, double lr) {
    int rc;
    if (!s || !grad || !(lr > 0)) return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    CK(cudaSetDevice(s->device));
    CK(cudaMemcpyAsync(s->g, grad, sizeof(float) * s->np, cudaMemcpyHostToDevice, s->st));
    if ((rc = adam(s, lr))) return rc;
    CK(cudaStreamSynchronize(s->st));
    return MB_OK;
}

int mb_sur_get_params(const mb_surrogate *s, float *params) {
    if (!s || !params) return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    CK(cudaSetDevice(s->device));
    CK(cudaMemcpyAsync(params, s->p, sizeof(float) * s->np, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return MB_OK;
}

int mb_sur_set_params(mb_surrogate *s, const float *params) {
    if (!s || !params) return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    CK(cudaSetDevice(s->device));
    CK(cudaMemcpyAsync(s->p, params, sizeof(float) * s->np, cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    return MB_OK;
}

int mb_sur_get_norm(const mb_surrogate *s, float *mean, float *istd, double *tmean, double *tstd) {
    if (!s) return mb_handle_fail(MB_ERR_ARG, "null handle");
    CK(cudaSetDevice(s->device));
    if (mean) CK(cudaMemcpyAsync(mean, s->mean, sizeof(float) * s->nin, cudaMemcpyDeviceToHost, s->st));
    if (istd) CK(cudaMemcpyAsync(istd, s->istd, sizeof(float) * s->nin, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (tmean) *tmean = s->tmean;
    if (tstd) *tstd = s->tstd;
    return MB_OK;
}
