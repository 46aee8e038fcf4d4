/*
 * maise_surrogate.h -- surrogate screen for EA offspring (B200).
 *
 * None of these entry points has a counterpart in the reference: MAISE's EA
 * relaxes every offspring (RELX_INT / RELX_TR, src/emod.c:521-757) before
 * ranking them by enthalpy (RANK_TR, src/emod.c:304-393).  The screen sits
 * between offspring creation and that relaxation: it predicts each
 * offspring's relaxed enthalpy per atom from its unrelaxed structure, and
 * only the best-ranked fraction is relaxed.  Every kept structure is still
 * relaxed by the full method, which also judges the screen's ranking.
 *
 * Features: per-species-pair radial histograms, the analogue of the
 * reference's RDF (src/cell.c:369-417) -- Gaussian-smeared pair distances
 * with a cosine taper, species(j) >= species(i), same-species halved --
 * at nbins bins up to rmax, divided by the atom count.
 * Model: FP32 MLP nin -> h1 -> h2 -> h3 -> 1 with SiLU, nin = nbins x
 * nspc (nspc + 1) / 2, trained by Adam on squared error of standardised
 * features and targets.  Back-propagation is the chain rule DE_ANN_PARA
 * (src/nmlp.c:292-354) applies to the potential's network.
 *
 * Parameters are one flat FP32 vector: for each layer W[out][in] row-major
 * followed by b[out].  All arrays are host arrays unless named d_*.  Every
 * call returns MB_OK or an MB_ERR_* code of maise_b200.h; mb_last_error()
 * gives the message.
 */
#ifndef MAISE_SURROGATE_H
#define MAISE_SURROGATE_H

#include "maise_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mb_surrogate mb_surrogate;

/* A new network on `device`: histograms of nbins bins up to rmax (A) with
 * Gaussian width sigma (A) for nspc species (<= 4), hidden widths h1, h2, h3,
 * weights N(0, 1/fan_in) from `seed`, zero biases. */
int mb_sur_open(int device, int nspc, int nbins, double rmax, double sigma, int h1, int h2, int h3, unsigned seed,
                mb_surrogate **out);
void mb_sur_close(mb_surrogate *s);
/* input width and parameter count */
int mb_sur_info(const mb_surrogate *s, int *nin, long *nparams);

/* Histogram features of S periodic structures (nat[s] atoms each, at most
 * 256; species atmn, Cartesian x and lattice rows lat[9 S] concatenated):
 * feat[S][nin]. */
int mb_sur_features(mb_surrogate *s, int S, const int *nat, const int *atmn, const double *lat, const double *x,
                    float *feat);

/* Train on S rows feat[S][nin] with targets y[S] (relaxed enthalpy per
 * atom, eV): the feature and target standardisation is fixed from these
 * rows, then `epochs` passes of Adam (learning rate lr, beta 0.9/0.999,
 * eps 1e-8) over minibatches of `batch` rows, shuffled each epoch from
 * `seed`.  loss[epochs] (may be NULL) receives each epoch's mean loss on the
 * standardised scale.  Calling it again continues from the current
 * parameters (the standardisation is recomputed). */
int mb_sur_fit(mb_surrogate *s, int S, const float *feat, const double *y, int epochs, int batch, double lr,
               unsigned seed, float *loss);

/* Predicted relaxed enthalpy per atom (eV) of S feature rows. */
int mb_sur_predict(mb_surrogate *s, int S, const float *feat, double *pred);

/* Features and prediction in one call, the features staying on the GPU. */
int mb_sur_screen(mb_surrogate *s, int S, const int *nat, const int *atmn, const double *lat, const double *x,
                  double *pred);

/* Checks of the training kernels on raw network inputs (no
 * standardisation): loss = mean((net(x) - t)^2) over B rows x[B][nin] and its
 * gradient grad[nparams]; and one Adam step with a given gradient (the
 * step count advances by one). */
int mb_sur_loss_grad(mb_surrogate *s, int B, const float *x, const float *t, double *loss, float *grad);
int mb_sur_adam_step(mb_surrogate *s, const float *grad, double lr);

int mb_sur_get_params(const mb_surrogate *s, float *params);
int mb_sur_set_params(mb_surrogate *s, const float *params);
/* the standardisation fixed by the last mb_sur_fit: mean[nin], istd[nin]
 * (1/std with a variance floor of 1e-6), target mean and std */
int mb_sur_get_norm(const mb_surrogate *s, float *mean, float *istd, double *tmean, double *tstd);

#ifdef __cplusplus
}
#endif
#endif
