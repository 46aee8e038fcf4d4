/*
 * maise_train.h -- C-ABI of the GPU training of MAISE's per-species neural
 * networks (the objective of tot_err_gsl and the gradient of dfunc_gsl /
 * DE_ANN_PARA, src/nmin.c:93-305 and src/nmlp.c:292-354, minimised as
 * MLP_MIN does, src/nmin.c:314-445).
 *
 * A training set is S structures with descriptors G (one row of D values per
 * atom, the reference's Cn, e.g. from mb_descriptors), species, reference
 * energies and weights.  Parameters are one vector V in the reference's V2W
 * order (src/nmlp.c:591-608): per species the biases b0[h1], b1[h2], b2[1],
 * then the weights W0[h1][D], W1[h2][h1], W2[1][h2]; hidden layers tanh,
 * output linear; the inputs are scaled as the model file's range table says,
 * x = (G - Rmin) * DR (rmin, dr: [nspc][D]), so a trained V is written to a
 * model file with that same table.
 */
#ifndef MAISE_TRAIN_H
#define MAISE_TRAIN_H

#include "maise_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define MB_TRAIN_MAXH 32 /* hidden-layer width */

typedef struct mb_train mb_train;

/* Upload a training set to CUDA device `device`.  nat[S] atoms per
 * structure, atmn/G rows per atom in structure order, E_ref[S] energies
 * (eV), weight[S] per-structure weights (NULL: all 1), WE the energy weight
 * and LREG the L2 regularisation of the reference's setup. */
int mb_train_open(int device, int S, const int *nat, const int *atmn, int nspc, int D, int h1, int h2,
                  const double *G, const double *rmin, const double *dr, const double *E_ref, const double *weight,
                  double WE, double LREG, mb_train **out);
int mb_train_close(mb_train *t);

/* Number of parameters (nspc * (h1 + h2 + 1 + h1 D + h2 h1 + h2)). */
int mb_train_info(const mb_train *t, int *nparams);

/* Objective RT = WE sum_s w_s ((E_s - E(s)) / N_s)^2 / S + LREG |V|^2 at V
 * (plus the force term once mb_train_set_forces was called), and (if
 * grad != NULL) its gradient; E_pred[S] (may be NULL) receives the
 * predicted energies E(s). */
int mb_train_eval(mb_train *t, const double *V, double *RT, double *grad, double *E_pred);

/* Force training (the reference's EFS 1 and 3, tot_err_gsl with
 * FRC_ANN_PARA and DF_ANN_PARA, src/nmin.c:111-132, src/nmlp.c:29-290):
 * NF marked atoms f_atom[NF] (rows of the training set's atoms) with
 * reference forces F_ref[3 NF] (eV/A) and their derivative blocks, marked
 * atom i owning blocks blk_off[i] .. blk_off[i+1]-1: block b is dG_o/dx_i
 * of owner atom blk_atom[b] (an atom of the same structure; the self block
 * has o = i), Fn[b][D][3] as the descriptor files hold it (dG/dx in the
 * descriptors' own scale).  scale_blocks = 1 puts the blocks on the
 * network's input scale, Fn[b][l] * dr[s_o][l], as ADJT_LNK does for EFS 1
 * (src/nmod.c:244-259; dr as in mb_train_open); 0 takes them as given
 * (ADJT_LNK leaves them unscaled for EFS 3).  After this call the objective
 * adds WF sum_s w_s sum_{i in s} |F_i - f_i|^2 / S and its gradient.
 * Once per trainer; MB_ERR_ARG if a block's owner lies outside its marked
 * atom's structure. */
int mb_train_set_forces(mb_train *t, int NF, const int *f_atom, const double *F_ref, const int *blk_off,
                        const int *blk_atom, const double *Fn, int scale_blocks, const double *dr, double WF);

/* Predicted forces f_pred[3 NF] of the marked atoms at V and (RF, may be
 * NULL) sum_s w_s sum_i |F_i - f_i|^2. */
int mb_train_eval_forces(mb_train *t, const double *V, double *f_pred, double *RF);

/* Minimise RT from V (updated in place) by BFGS with Fletcher's line search
 * (initial step 0.01, line tolerance 1e-5), at most mitr iterations or until
 * |grad| < gtol; RT and iters (may be NULL) receive the final objective and
 * the iterations taken. */
int mb_train_fit(mb_train *t, double *V, int mitr, double gtol, double *RT, int *iters);

#ifdef __cplusplus
}
#endif
#endif
