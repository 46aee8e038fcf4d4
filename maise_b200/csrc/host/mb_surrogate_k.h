/*
 * mb_surrogate_k.h -- launchers of the surrogate kernels (mb_surrogate.cu),
 * called by the host side in mb_surrogate.c.  All return a cudaError_t
 * value (0 on success).
 */
#ifndef MB_SURROGATE_K_H
#define MB_SURROGATE_K_H

#ifdef __cplusplus
extern "C" {
#endif

#define SUR_MAX_ATOMS 256  /* atoms per structure in the histogram kernel */
#define SUR_MAX_SPC 4      /* species (10 pair histograms) */
#define SUR_MAX_IMG 6      /* periodic images per direction and side */
#define SUR_VAR_FLOOR 1e-6 /* added to a feature's variance before 1/std */

/* GEMM epilogues */
#define SUR_EP_STORE 0     /* C = A B */
#define SUR_EP_BIAS 1      /* C = A B + bias */
#define SUR_EP_BIAS_SILU 2 /* Z = A B + bias, C = SiLU(Z) */
#define SUR_EP_DSILU 3     /* C = (A B) * SiLU'(Zp) */

int surk_rdf(int S, const int *off, const int *spc, const double *lat, const double *x, int nspc, int nbins,
             double rmax, double sigma, float *feat, int *status, void *stream);
int surk_gemm(int ta, int tb, int ep, int M, int N, int K, const float *A, int lda, const float *B, int ldb, float *C,
              int ldc, const float *bias, float *Z, const float *Zp, void *stream);
int surk_colsum(int B, int O, const float *dZ, float *out, void *stream);
int surk_mse(int B, const float *y, const float *t, float *dy, double *loss, void *stream);
int surk_adam(long n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2, float eps, float c1,
              float c2, void *stream);
int surk_gather(int B, int F, const int *idx, const float *X, const float *mean, const float *istd, float *out,
                const float *T, float tmean, float tistd, float *tout, void *stream);
int surk_colstats(int S, int F, const float *X, float *mean, float *istd, void *stream);

#ifdef __cplusplus
}
#endif
#endif
