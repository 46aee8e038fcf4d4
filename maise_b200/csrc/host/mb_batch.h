/* mb_batch.h -- launcher of the persistent population relax (mb_batch.cu). */
#ifndef MB_BATCH_H
#define MB_BATCH_H
#include "../mb_internal.h"
#ifdef __cplusplus
extern "C" {
#endif
int mbk_relax_batch(const mb_model *m, int S, const int *d_nat, const int *d_off, const int *d_spc,
                    const int *d_order, double *d_lat, double *d_x, double p_ev, double urep, int rlxt, int mitr, double fmax, double *d_H, int *d_iters,
                    int *d_status, double *d_frc, double *d_str, void *stream, long long *evals_out, float *ms_out);
#ifdef __cplusplus
}
#endif
#endif
