/*
 * mb_bfgs.h -- dense-inverse-Hessian BFGS with Fletcher's line search.
 *
 * Written from the published algorithms: the BFGS inverse update of
 * Nocedal & Wright, "Numerical Optimization" (2nd ed.) eqs. 6.17 and 6.20,
 * and the bracketing/sectioning line search of Fletcher, "Practical Methods
 * of Optimization" (2nd ed.), Algorithms 2.6.2 and 2.6.4, with sigma = the
 * caller's tolerance, rho = 0.01, tau1 = 9, tau2 = 0.05, tau3 = 0.5.
 *
 * It plays the role of GSL 1.16's vector_bfgs2 minimiser used by the
 * reference relaxation (src/cmin.c:214-276: step size 0.01, tolerance
 * 0.001).  GSL's code is not used; trajectories are not iterate-identical
 * to GSL's, final minima are.
 */
#ifndef MB_BFGS_H
#define MB_BFGS_H

#ifdef __cplusplus
extern "C" {
#endif

/* energy only at x; the callee may rewrite x in place (e.g. wrap fractional
 * coordinates back into the cell, as src/cmin.c:90-105 does). */
typedef double (*mb_fn_f)(void *ctx, double *x);
/* energy and gradient at x; same in-place rule. */
typedef double (*mb_fn_fg)(void *ctx, double *x, double *g);

enum { MB_BFGS_OK = 0, MB_BFGS_NOPROG = 27, MB_BFGS_EBADFUNC = 9 };

typedef struct {
    int n;
    double *x, *g, *H, *p, *xt, *gt, *xa, *ga, *tmp;
    double f, fprev, step0, sigma;
    int first;
    long nf, nfg;            /* energy-only and energy+gradient evaluations */
    mb_fn_f fn_f;
    mb_fn_fg fn_fg;
    void *ctx;
} mb_bfgs;

/* Allocates state, copies x0 and evaluates f and g there. */
int mb_bfgs_init(mb_bfgs *s, int n, const double *x0, double step, double tol, mb_fn_f f, mb_fn_fg fg, void *ctx);
/* One quasi-Newton iteration: line search along -H g, then the BFGS update.
 * Returns MB_BFGS_OK, or MB_BFGS_NOPROG when no acceptable step exists. */
int mb_bfgs_iterate(mb_bfgs *s);
/* Resets the inverse Hessian to the identity. */
void mb_bfgs_restart(mb_bfgs *s);
void mb_bfgs_free(mb_bfgs *s);

#ifdef __cplusplus
}
#endif
#endif
