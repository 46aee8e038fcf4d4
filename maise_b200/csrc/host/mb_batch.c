/*
 * mb_batch.c -- host side of the population relax: packs the structures,
 * launches the persistent kernel (mb_batch.cu) and returns the results.
 */
#include <cuda_runtime_api.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../../include/maise_b200.h"
#include "mb_batch.h"

#define MB_EV2GPA 160.2176565 /* src/util.c:8 */

/* the handle layout is private to mb_core.c; these accessors are defined there */
const mb_model *mb_handle_model(const mb_potential *p);
void *mb_handle_stream(mb_potential *p);
int mb_handle_device(const mb_potential *p);
int mb_handle_fail(int code, const char *msg);
void mb_handle_set_batch_stats(mb_potential *p, const long long *evals, float ms);

/* The population relax and the batched E/F/S share this: with frc/str set
 * the kernel also returns each structure's forces and virial at its final
 * state, and with keep_xyz = 0 the positions and lattices are not copied back. */
static int batch_run(mb_potential *pot, int S, const int *nat, const int *atmn, double *lat, double *x, double p_gpa,
                     double urep, int rlxt, int mitr, double fmax, double *H, int *iters, int *status, double *frc,
                     double *str, int keep_xyz) {
    int *off, *order, total = 0, s, rc = MB_OK;
    int *d_nat = NULL, *d_off = NULL, *d_spc = NULL, *d_iters = NULL, *d_status = NULL, *d_order = NULL;
    double *d_lat = NULL, *d_x = NULL, *d_H = NULL, *d_frc = NULL, *d_str = NULL;
    long long evals[4] = {0, 0, 0, 0}; /* evaluations, atom evaluations, pairs, triplets */
    float ms = 0.0f;
    const mb_model *m;
    void *st;
    cudaError_t e;
    if (!pot || S < 1 || !nat || !atmn || !lat || !x || !H || !iters || !status || !(fmax > 0) || mitr < 0)
        return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    if (!(rlxt == 2 || rlxt == 3)) return mb_handle_fail(MB_ERR_ARG, "batched relax supports RLXT 2 and 3");
    m = mb_handle_model(pot);
    off = (int *)malloc(sizeof(int) * (S + 1));
    for (s = 0; s < S; s++) {
        if (nat[s] < 1 || nat[s] > 64) {
            free(off);
            return mb_handle_fail(MB_ERR_ARG, "batched relax takes 1..64 atoms per structure");
        }
        off[s] = total;
        total += nat[s];
    }
    off[S] = total;
    for (s = 0; s < total; s++)
        if (atmn[s] < 0 || atmn[s] >= m->nspc) {
            free(off);
            return mb_handle_fail(MB_ERR_ARG, "species index out of range");
        }
    /* the persistent CTAs take structures largest first, so that the last
     * ones to start are small and the population finishes evenly */
    order = (int *)malloc(sizeof(int) * S);
    {
        int n, k = 0;
        for (n = 64; n >= 1; n--)
            for (s = 0; s < S; s++)
                if (nat[s] == n) order[k++] = s;
    }
    cudaSetDevice(mb_handle_device(pot));
    st = mb_handle_stream(pot);
    e = cudaMalloc((void **)&d_nat, sizeof(int) * S);
    if (!e) e = cudaMalloc((void **)&d_off, sizeof(int) * (S + 1));
    if (!e) e = cudaMalloc((void **)&d_spc, sizeof(int) * total);
    if (!e) e = cudaMalloc((void **)&d_iters, sizeof(int) * S);
    if (!e) e = cudaMalloc((void **)&d_status, sizeof(int) * S);
    if (!e) e = cudaMalloc((void **)&d_lat, sizeof(double) * 9 * S);
    if (!e) e = cudaMalloc((void **)&d_x, sizeof(double) * 3 * total);
    if (!e) e = cudaMalloc((void **)&d_H, sizeof(double) * S);
    if (!e) e = cudaMalloc((void **)&d_order, sizeof(int) * S);
    if (!e && frc) e = cudaMalloc((void **)&d_frc, sizeof(double) * 3 * total);
    if (!e && str) e = cudaMalloc((void **)&d_str, sizeof(double) * 6 * S);
    if (!e) e = cudaMemcpyAsync(d_order, order, sizeof(int) * S, cudaMemcpyHostToDevice, (cudaStream_t)st);
    if (!e) e = cudaMemcpyAsync(d_nat, nat, sizeof(int) * S, cudaMemcpyHostToDevice, (cudaStream_t)st);
    if (!e) e = cudaMemcpyAsync(d_off, off, sizeof(int) * (S + 1), cudaMemcpyHostToDevice, (cudaStream_t)st);
    if (!e) e = cudaMemcpyAsync(d_spc, atmn, sizeof(int) * total, cudaMemcpyHostToDevice, (cudaStream_t)st);
    if (!e) e = cudaMemcpyAsync(d_lat, lat, sizeof(double) * 9 * S, cudaMemcpyHostToDevice, (cudaStream_t)st);
    if (!e) e = cudaMemcpyAsync(d_x, x, sizeof(double) * 3 * total, cudaMemcpyHostToDevice, (cudaStream_t)st);
    if (e) {
        rc = mb_handle_fail(MB_ERR_CUDA, cudaGetErrorString(e));
        goto out;
    }
    e = (cudaError_t)mbk_relax_batch(m, S, d_nat, d_off, d_spc, d_order, d_lat, d_x, p_gpa / MB_EV2GPA, urep > 0 ? urep : 0.0,
                                     rlxt, mitr, fmax, d_H, d_iters, d_status, frc ? d_frc : NULL,
                                     frc ? d_str : NULL, st, evals, &ms);
    if (e == cudaErrorInvalidValue) {
        rc = mb_handle_fail(MB_ERR_MODEL, "batched relax needs a basis with <= 7 G4 exponents, zeta in {integers}, "
                                          "2 lambdas, <= 16 G2 functions and D <= 288");
        goto out;
    }
    if (e) {
        rc = mb_handle_fail(MB_ERR_CUDA, cudaGetErrorString(e));
        goto out;
    }
    e = cudaSuccess;
    if (keep_xyz) {
        e = cudaMemcpy(lat, d_lat, sizeof(double) * 9 * S, cudaMemcpyDeviceToHost);
        if (!e) e = cudaMemcpy(x, d_x, sizeof(double) * 3 * total, cudaMemcpyDeviceToHost);
    }
    if (!e && frc) e = cudaMemcpy(frc, d_frc, sizeof(double) * 3 * total, cudaMemcpyDeviceToHost);
    if (!e && frc && str) e = cudaMemcpy(str, d_str, sizeof(double) * 6 * S, cudaMemcpyDeviceToHost);
    if (!e) e = cudaMemcpy(H, d_H, sizeof(double) * S, cudaMemcpyDeviceToHost);
    if (!e) e = cudaMemcpy(iters, d_iters, sizeof(int) * S, cudaMemcpyDeviceToHost);
    if (!e) e = cudaMemcpy(status, d_status, sizeof(int) * S, cudaMemcpyDeviceToHost);
    if (e) rc = mb_handle_fail(MB_ERR_CUDA, cudaGetErrorString(e));
    mb_handle_set_batch_stats(pot, evals, ms);
out:
    cudaFree(d_nat); cudaFree(d_off); cudaFree(d_spc); cudaFree(d_iters); cudaFree(d_status);
    cudaFree(d_lat); cudaFree(d_x); cudaFree(d_H); cudaFree(d_order); cudaFree(d_frc); cudaFree(d_str);
    free(off);
    free(order);
    return rc;
}

int mb_relax_batch(mb_potential *pot, int S, const int *nat, const int *atmn, double *lat, double *x, double p_gpa,
                   double urep, int rlxt, int mitr, double fmax, double *H, int *iters, int *status) {
    return batch_run(pot, S, nat, atmn, lat, x, p_gpa, urep, rlxt, mitr, fmax, H, iters, status, NULL, NULL, 1);
}

int mb_efs_batch(mb_potential *pot, int S, const int *nat, const int *atmn, const double *lat, const double *x,
                 double p_gpa, double urep, double *H, double *frc, double *str) {
    int *iters, *status, rc;
    if (!frc || !H || S < 1) return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    iters = (int *)malloc(sizeof(int) * S);
    status = (int *)malloc(sizeof(int) * S);
    /* no iterations: the kernel evaluates each structure once; the
     * positions and lattices are read, not written back */
    rc = batch_run(pot, S, nat, atmn, (double *)lat, (double *)x, p_gpa, urep, 3, 0, 1.0, H, iters, status, frc, str,
                   0);
    if (!rc)
        for (int s = 0; s < S; s++)
            if (status[s] == 2) {
                rc = mb_handle_fail(MB_ERR_NEIGHBOURS, "a structure has more than 96 neighbours per atom");
                break;
            }
    free(iters);
    free(status);
    return rc;
}

int mb_evos_write(const char *evos_dir, int gen, int member, int N, int nspc, const int *spcz, const int *atmn,
                  const double *lat0, const double *x0, const double *lat, const double *x, double H, double E,
                  double p_gpa, const double *frc, const double *str, int iters);

int mb_evos_relax(mb_potential *pot, const char *evos_dir, int gen, int p0, int S, const int *nat, const int *atmn,
                  double *lat, double *x, double p_gpa, double urep, int rlxt, int mitr, double fmax, double *H,
                  int *iters, int *status) {
    const mb_model *m;
    double *lat0, *x0, *frc, *str;
    int total = 0, s, rc, off = 0;
    if (!pot || !evos_dir || S < 1 || !nat || !atmn || !lat || !x || !H || !iters || !status || p0 < 0 || gen < 0)
        return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    for (s = 0; s < S; s++) total += nat[s] > 0 ? nat[s] : 0;
    m = mb_handle_model(pot);
    lat0 = (double *)malloc(sizeof(double) * 9 * S);
    x0 = (double *)malloc(sizeof(double) * 3 * total);
    frc = (double *)malloc(sizeof(double) * 3 * total);
    str = (double *)malloc(sizeof(double) * 6 * S);
    if (!lat0 || !x0 || !frc || !str) {
        free(lat0); free(x0); free(frc); free(str);
        return mb_handle_fail(MB_ERR_ARG, "out of memory");
    }
    memcpy(lat0, lat, sizeof(double) * 9 * S);
    memcpy(x0, x, sizeof(double) * 3 * total);
    rc = batch_run(pot, S, nat, atmn, lat, x, p_gpa, urep, rlxt, mitr, fmax, H, iters, status, frc, str, 1);
    for (s = 0; s < S && rc == MB_OK; s++) {
        const double *L = lat + 9 * s;
        const double V = fabs(L[0] * L[4] * L[8] + L[2] * L[3] * L[7] + L[1] * L[5] * L[6] - L[0] * L[5] * L[7] -
                              L[1] * L[3] * L[8] - L[2] * L[4] * L[6]);
        const double E = H[s] - p_gpa / MB_EV2GPA * V;
        rc = mb_evos_write(evos_dir, gen, p0 + s, nat[s], m->nspc, m->spcz, atmn + off, lat0 + 9 * s, x0 + 3 * off,
                           L, x + 3 * off, H[s], E, p_gpa, frc + 3 * off, str + 6 * s, iters[s]);
        off += nat[s];
    }
    free(lat0); free(x0); free(frc); free(str);
    return rc;
}
