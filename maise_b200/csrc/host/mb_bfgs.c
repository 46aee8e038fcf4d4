/*
 * mb_bfgs.c -- BFGS quasi-Newton minimiser with Fletcher's line search.
 * See mb_bfgs.h for the published algorithms this follows.
 */
#include "mb_bfgs.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define LS_RHO 0.01
#define LS_TAU1 9.0
#define LS_TAU2 0.05
#define LS_TAU3 0.5
#define LS_MAX_BRACKET 40
#define LS_MAX_SECTION 60

static double dotn(int n, const double *a, const double *b) {
    double r = 0.0;
    int i;
    for (i = 0; i < n; i++) r += a[i] * b[i];
    return r;
}

static void set_identity(int n, double *H, double scale) {
    int i;
    memset(H, 0, sizeof(double) * (size_t)n * n);
    for (i = 0; i < n; i++) H[(size_t)i * n + i] = scale;
}

int mb_bfgs_init(mb_bfgs *s, int n, const double *x0, double step, double tol, mb_fn_f f, mb_fn_fg fg, void *ctx) {
    memset(s, 0, sizeof(*s));
    s->n = n;
    s->x = (double *)malloc(sizeof(double) * n);
    s->g = (double *)malloc(sizeof(double) * n);
    s->p = (double *)malloc(sizeof(double) * n);
    s->xt = (double *)malloc(sizeof(double) * n);
    s->gt = (double *)malloc(sizeof(double) * n);
    s->xa = (double *)malloc(sizeof(double) * n);
    s->ga = (double *)malloc(sizeof(double) * n);
    s->tmp = (double *)malloc(sizeof(double) * n);
    s->H = (double *)malloc(sizeof(double) * (size_t)n * n);
    if (!s->x || !s->g || !s->p || !s->xt || !s->gt || !s->xa || !s->ga || !s->tmp || !s->H) return -1;
    memcpy(s->x, x0, sizeof(double) * n);
    s->step0 = step;
    s->sigma = tol;
    s->fn_f = f;
    s->fn_fg = fg;
    s->ctx = ctx;
    s->first = 1;
    set_identity(n, s->H, 1.0);
    s->f = fg(ctx, s->x, s->g);
    s->nfg++;
    s->fprev = s->f;
    return 0;
}

void mb_bfgs_restart(mb_bfgs *s) {
    set_identity(s->n, s->H, 1.0);
    s->first = 1;
}

void mb_bfgs_free(mb_bfgs *s) {
    free(s->x); free(s->g); free(s->p); free(s->xt); free(s->gt);
    free(s->xa); free(s->ga); free(s->tmp); free(s->H);
    memset(s, 0, sizeof(*s));
}

/* Minimiser over [lo,hi] of the cubic Hermite interpolant through
 * (a,fa,da) and (b,fb,db); if db is unknown (has_db == 0) the quadratic
 * through fa, da, fb is used.  Fletcher, sec. 2.6. */
static double interp_min(double a, double fa, double da, double b, double fb, double db, int has_db, double lo,
                         double hi) {
    double w = b - a, zlo, zhi, c0 = fa, c1 = da * w, c2, c3, best, fbest, z;
    double cand[4];
    int nc = 0, k;
    if (w == 0.0) return a;
    zlo = (lo - a) / w;
    zhi = (hi - a) / w;
    if (zlo > zhi) { double t = zlo; zlo = zhi; zhi = t; }
    if (has_db) {
        c2 = 3.0 * (fb - fa) - 2.0 * c1 - db * w;
        c3 = c1 + db * w - 2.0 * (fb - fa);
    } else {
        c2 = fb - fa - c1;
        c3 = 0.0;
    }
    cand[nc++] = zlo;
    cand[nc++] = zhi;
    if (c3 != 0.0) {
        /* roots of c1 + 2 c2 z + 3 c3 z^2 */
        double disc = 4.0 * c2 * c2 - 12.0 * c3 * c1;
        if (disc >= 0.0) {
            double sq = sqrt(disc);
            double q = -0.5 * (2.0 * c2 + (c2 >= 0.0 ? sq : -sq));
            if (q != 0.0) cand[nc++] = q / (3.0 * c3);
            cand[nc++] = c1 / (q != 0.0 ? q : -DBL_MIN);
        }
    } else if (c2 > 0.0) {
        cand[nc++] = -c1 / (2.0 * c2);
    }
    best = zlo;
    fbest = DBL_MAX;
    for (k = 0; k < nc; k++) {
        double fz;
        z = cand[k];
        if (!(z >= zlo && z <= zhi)) continue;
        fz = c0 + z * (c1 + z * (c2 + z * c3));
        if (fz < fbest) { fbest = fz; best = z; }
    }
    return a + best * w;
}

/* phi(alpha) at xt = x + alpha p; energy only */
static double phi_f(mb_bfgs *s, double alpha) {
    int i;
    for (i = 0; i < s->n; i++) s->xt[i] = s->x[i] + alpha * s->p[i];
    s->nf++;
    return s->fn_f(s->ctx, s->xt);
}

/* phi and phi' at xt = x + alpha p; gradient left in gt */
static double phi_fg(mb_bfgs *s, double alpha, double *dphi) {
    int i;
    double f;
    for (i = 0; i < s->n; i++) s->xt[i] = s->x[i] + alpha * s->p[i];
    s->nfg++;
    f = s->fn_fg(s->ctx, s->xt, s->gt);
    *dphi = dotn(s->n, s->gt, s->p);
    return f;
}

/* Fletcher line search.  On success returns 1 with the accepted point in
 * xt/gt, its value in *fout and step in *aout. */
static int line_search(mb_bfgs *s, double alpha1, double phi0, double dphi0, double *aout, double *fout) {
    const double rho = LS_RHO, sigma = s->sigma;
    double ap = 0.0, fp = phi0, dp = dphi0; /* previous trial (starts at 0) */
    double a, fa, da, b, fb, db = 0.0, alpha = alpha1;
    int has_db = 0, it, n = s->n;
    /* gradient at the lower end "a" of a bracket is kept in xa/ga */
    memcpy(s->xa, s->x, sizeof(double) * n);
    memcpy(s->ga, s->g, sizeof(double) * n);

    for (it = 0; it < LS_MAX_BRACKET; it++) {
        double f = phi_f(s, alpha), d;
        if (!isfinite(f)) return 0;
        if (f > phi0 + rho * alpha * dphi0 || (it > 0 && f >= fp)) {
            a = ap; fa = fp; da = dp;
            b = alpha; fb = f; has_db = 0;
            goto section;
        }
        f = phi_fg(s, alpha, &d);
        if (fabs(d) <= -sigma * dphi0) { *aout = alpha; *fout = f; return 1; }
        if (d >= 0.0) {
            a = alpha; fa = f; da = d;
            memcpy(s->xa, s->xt, sizeof(double) * n);
            memcpy(s->ga, s->gt, sizeof(double) * n);
            b = ap; fb = fp; db = dp; has_db = 1;
            goto section;
        }
        {
            double lo = 2.0 * alpha - ap, hi = alpha + LS_TAU1 * (alpha - ap);
            double next = interp_min(ap, fp, dp, alpha, f, d, 1, lo, hi);
            ap = alpha; fp = f; dp = d;
            memcpy(s->xa, s->xt, sizeof(double) * n);
            memcpy(s->ga, s->gt, sizeof(double) * n);
            alpha = next;
        }
    }
    return 0;

section:
    for (it = 0; it < LS_MAX_SECTION; it++) {
        double lo = a + LS_TAU2 * (b - a), hi = b - LS_TAU3 * (b - a), f, d;
        alpha = interp_min(a, fa, da, b, fb, db, has_db, lo, hi);
        f = phi_f(s, alpha);
        if (!isfinite(f)) break;
        if (f > phi0 + rho * alpha * dphi0 || f >= fa) {
            b = alpha; fb = f; has_db = 0;
        } else {
            f = phi_fg(s, alpha, &d);
            if (fabs(d) <= -sigma * dphi0) { *aout = alpha; *fout = f; return 1; }
            if ((b - a) * d >= 0.0) { b = a; fb = fa; db = da; has_db = 1; }
            a = alpha; fa = f; da = d;
            memcpy(s->xa, s->xt, sizeof(double) * n);
            memcpy(s->ga, s->gt, sizeof(double) * n);
        }
        /* interval shrunk to round-off: the best point found so far stands */
        if (fabs((a - b) * da) <= 4.0 * DBL_EPSILON * (fabs(phi0) + 1.0)) break;
    }
    if (a > 0.0 && fa < phi0) {
        memcpy(s->xt, s->xa, sizeof(double) * n);
        memcpy(s->gt, s->ga, sizeof(double) * n);
        *aout = a;
        *fout = fa;
        return 1;
    }
    return 0;
}

int mb_bfgs_iterate(mb_bfgs *s) {
    int n = s->n, i, j;
    double dphi0, pnorm, alpha1, alpha, fnew, sy, yy;
    double *Hy = s->tmp;
    /* p = -H g */
    for (i = 0; i < n; i++) {
        double t = 0.0;
        for (j = 0; j < n; j++) t += s->H[(size_t)i * n + j] * s->g[j];
        s->p[i] = -t;
    }
    dphi0 = dotn(n, s->g, s->p);
    if (!(dphi0 < 0.0)) {
        /* not a descent direction: restart along the steepest descent */
        mb_bfgs_restart(s);
        for (i = 0; i < n; i++) s->p[i] = -s->g[i];
        dphi0 = dotn(n, s->g, s->p);
    }
    if (!(dphi0 < 0.0)) return MB_BFGS_NOPROG;
    pnorm = sqrt(dotn(n, s->p, s->p));
    if (s->first)
        alpha1 = s->step0 / pnorm;
    else {
        alpha1 = 2.0 * (s->f - s->fprev) / dphi0;
        if (!(alpha1 > 0.0) || alpha1 > 1.0) alpha1 = 1.0;
    }
    if (!line_search(s, alpha1, s->f, dphi0, &alpha, &fnew)) return MB_BFGS_NOPROG;

    /* s_k = alpha p (stored in p), y_k = g_new - g (stored in g) */
    for (i = 0; i < n; i++) {
        s->p[i] *= alpha;
        s->g[i] = s->gt[i] - s->g[i];
    }
    sy = dotn(n, s->p, s->g);
    yy = dotn(n, s->g, s->g);
    if (sy > 0.0) {
        double yHy, c1;
        if (s->first) set_identity(n, s->H, sy / yy);
        for (i = 0; i < n; i++) {
            double t = 0.0;
            for (j = 0; j < n; j++) t += s->H[(size_t)i * n + j] * s->g[j];
            Hy[i] = t;
        }
        yHy = dotn(n, s->g, Hy);
        c1 = (sy + yHy) / (sy * sy);
        for (i = 0; i < n; i++)
            for (j = 0; j < n; j++)
                s->H[(size_t)i * n + j] += c1 * s->p[i] * s->p[j] - (Hy[i] * s->p[j] + s->p[i] * Hy[j]) / sy;
    }
    memcpy(s->x, s->xt, sizeof(double) * n);
    memcpy(s->g, s->gt, sizeof(double) * n);
    s->fprev = s->f;
    s->f = fnew;
    s->first = 0;
    return MB_BFGS_OK;
}
