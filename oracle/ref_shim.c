/*
 * ref_shim.c -- stand-ins for the third-party symbols the reference sources
 * link against, so that the reference can be compiled here as a CPU
 * oracle.  TEST INFRASTRUCTURE ONLY (see oracle/Makefile).
 *
 * GSL 1.16 (pinned by the reference's dep-gsl:2-3) is not present in this
 * image: only its headers ship under lib/include/gsl.  This file is compiled
 * against those headers so the struct layouts seen by src/cmin.c match, and
 * provides:
 *   - gsl_vector_{alloc,free,get,set} and gsl_strerror;
 *   - the gsl_multimin_fdfminimizer API used by CELL_MIN (src/cmin.c:177-301),
 *     backed by the project's BFGS with Fletcher's line search
 *     (maise_b200/csrc/host/mb_bfgs.c, written from the published
 *     algorithm -- GSL's own code is not used);
 *   - gsl_multimin_test_size (GSL manual: success iff size < epsabs);
 *   - a 3x3 symmetric eigen-solve behind gsl_eigen_nonsymmv for the
 *     particle volume of 0D cells (src/nutl.c:846-898 via src/util.c:80-122);
 *     only the eigenvalue product is used there;
 * and abort stubs for everything else (phonons, training, symmetry), which
 * the energy/force/stress, relax and MD paths never reach.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <gsl/gsl_eigen.h>
#include <gsl/gsl_errno.h>
#include <gsl/gsl_matrix.h>
#include <gsl/gsl_multimin.h>
#include <gsl/gsl_vector.h>

#include "../maise_b200/csrc/host/mb_bfgs.h"

static void shim_abort(const char *name) {
    fprintf(stderr, "oracle shim: %s is not available in this build\n", name);
    abort();
}

/* ---------------- vectors ---------------- */
gsl_vector *gsl_vector_alloc(const size_t n) {
    gsl_vector *v = (gsl_vector *)calloc(1, sizeof(gsl_vector));
    v->size = n;
    v->stride = 1;
    v->data = (double *)calloc(n ? n : 1, sizeof(double));
    v->owner = 1;
    return v;
}
void gsl_vector_free(gsl_vector *v) {
    if (!v) return;
    if (v->owner) free(v->data);
    free(v);
}
double gsl_vector_get(const gsl_vector *v, const size_t i) { return v->data[i * v->stride]; }
void gsl_vector_set(gsl_vector *v, const size_t i, double x) { v->data[i * v->stride] = x; }

const char *gsl_strerror(const int gsl_errno) {
    switch (gsl_errno) {
        case GSL_SUCCESS: return "success";
        case GSL_CONTINUE: return "the iteration has not converged yet";
        case GSL_ENOPROG: return "iteration is not making progress towards solution";
        default: return "error";
    }
}

/* ---------------- minimiser ---------------- */
typedef struct {
    mb_bfgs b;
    gsl_multimin_function_fdf *fdf;
    gsl_vector *view;  /* wraps arrays handed to the user callbacks */
    gsl_vector *gview;
    int ready;
} shim_state;

static double shim_f(void *ctx, double *x) {
    shim_state *st = (shim_state *)ctx;
    st->view->data = x;
    return st->fdf->f(st->view, st->fdf->params);
}
static double shim_fg(void *ctx, double *x, double *g) {
    shim_state *st = (shim_state *)ctx;
    double f;
    st->view->data = x;
    st->gview->data = g;
    f = st->fdf->f(st->view, st->fdf->params);
    st->fdf->df(st->view, st->fdf->params, st->gview);
    return f;
}

static int shim_type_alloc(void *state, size_t n) { (void)state; (void)n; return GSL_SUCCESS; }
static int shim_type_set(void *state, gsl_multimin_function_fdf *fdf, const gsl_vector *x, double *f,
                         gsl_vector *gradient, double step_size, double tol) {
    (void)state; (void)fdf; (void)x; (void)f; (void)gradient; (void)step_size; (void)tol;
    return GSL_SUCCESS;
}
static int shim_type_iterate(void *state, gsl_multimin_function_fdf *fdf, gsl_vector *x, double *f,
                             gsl_vector *gradient, gsl_vector *dx) {
    (void)state; (void)fdf; (void)x; (void)f; (void)gradient; (void)dx;
    return GSL_SUCCESS;
}
static int shim_type_restart(void *state) { (void)state; return GSL_SUCCESS; }
static void shim_type_free(void *state) { (void)state; }

static const gsl_multimin_fdfminimizer_type shim_bfgs_type = {
    "bfgs (project restatement)", sizeof(shim_state), shim_type_alloc, shim_type_set,
    shim_type_iterate,           shim_type_restart,  shim_type_free};

/* All four reference optimiser choices map onto the same BFGS here. */
const gsl_multimin_fdfminimizer_type *gsl_multimin_fdfminimizer_vector_bfgs2 = &shim_bfgs_type;
const gsl_multimin_fdfminimizer_type *gsl_multimin_fdfminimizer_conjugate_pr = &shim_bfgs_type;
const gsl_multimin_fdfminimizer_type *gsl_multimin_fdfminimizer_conjugate_fr = &shim_bfgs_type;
const gsl_multimin_fdfminimizer_type *gsl_multimin_fdfminimizer_steepest_descent = &shim_bfgs_type;

gsl_multimin_fdfminimizer *gsl_multimin_fdfminimizer_alloc(const gsl_multimin_fdfminimizer_type *T, size_t n) {
    gsl_multimin_fdfminimizer *s = (gsl_multimin_fdfminimizer *)calloc(1, sizeof(*s));
    shim_state *st = (shim_state *)calloc(1, sizeof(shim_state));
    s->type = T;
    s->x = gsl_vector_alloc(n);
    s->gradient = gsl_vector_alloc(n);
    s->dx = gsl_vector_alloc(n);
    st->view = (gsl_vector *)calloc(1, sizeof(gsl_vector));
    st->gview = (gsl_vector *)calloc(1, sizeof(gsl_vector));
    st->view->size = st->gview->size = n;
    st->view->stride = st->gview->stride = 1;
    s->state = st;
    return s;
}

int gsl_multimin_fdfminimizer_set(gsl_multimin_fdfminimizer *s, gsl_multimin_function_fdf *fdf, const gsl_vector *x,
                                  double step_size, double tol) {
    shim_state *st = (shim_state *)s->state;
    size_t n = x->size, i;
    double *x0 = (double *)malloc(sizeof(double) * n);
    for (i = 0; i < n; i++) x0[i] = gsl_vector_get(x, i);
    if (st->ready) mb_bfgs_free(&st->b);
    st->fdf = fdf;
    s->fdf = fdf;
    if (mb_bfgs_init(&st->b, (int)n, x0, step_size, tol, shim_f, shim_fg, st)) { free(x0); return GSL_ENOMEM; }
    st->ready = 1;
    free(x0);
    s->f = st->b.f;
    memcpy(s->x->data, st->b.x, sizeof(double) * n);
    memcpy(s->gradient->data, st->b.g, sizeof(double) * n);
    return GSL_SUCCESS;
}

int gsl_multimin_fdfminimizer_iterate(gsl_multimin_fdfminimizer *s) {
    shim_state *st = (shim_state *)s->state;
    size_t n = s->x->size, i;
    int rc = mb_bfgs_iterate(&st->b);
    for (i = 0; i < n; i++) s->dx->data[i] = st->b.x[i] - s->x->data[i];
    s->f = st->b.f;
    memcpy(s->x->data, st->b.x, sizeof(double) * n);
    memcpy(s->gradient->data, st->b.g, sizeof(double) * n);
    return rc == MB_BFGS_OK ? GSL_SUCCESS : GSL_ENOPROG;
}

int gsl_multimin_fdfminimizer_restart(gsl_multimin_fdfminimizer *s) {
    mb_bfgs_restart(&((shim_state *)s->state)->b);
    return GSL_SUCCESS;
}

void gsl_multimin_fdfminimizer_free(gsl_multimin_fdfminimizer *s) {
    shim_state *st;
    if (!s) return;
    st = (shim_state *)s->state;
    if (st->ready) mb_bfgs_free(&st->b);
    free(st->view);
    free(st->gview);
    free(st);
    gsl_vector_free(s->x);
    gsl_vector_free(s->gradient);
    gsl_vector_free(s->dx);
    free(s);
}

int gsl_multimin_test_size(const double size, double epsabs) {
    if (epsabs < 0.0) return GSL_EBADTOL;
    return size < epsabs ? GSL_SUCCESS : GSL_CONTINUE;
}

int gsl_multimin_test_gradient(const gsl_vector *g, double epsabs) {
    double n2 = 0.0;
    size_t i;
    for (i = 0; i < g->size; i++) n2 += gsl_vector_get(g, i) * gsl_vector_get(g, i);
    return sqrt(n2) < epsabs ? GSL_SUCCESS : GSL_CONTINUE;
}

/* ---------------- 3x3 eigen-solve for the particle volume ---------------- */
gsl_matrix_view gsl_matrix_view_array(double *base, const size_t n1, const size_t n2) {
    gsl_matrix_view v;
    memset(&v, 0, sizeof(v));
    v.matrix.size1 = n1;
    v.matrix.size2 = n2;
    v.matrix.tda = n2;
    v.matrix.data = base;
    return v;
}
gsl_vector_complex *gsl_vector_complex_alloc(const size_t n) {
    gsl_vector_complex *v = (gsl_vector_complex *)calloc(1, sizeof(*v));
    v->size = n;
    v->stride = 1;
    v->data = (double *)calloc(2 * n, sizeof(double));
    v->owner = 1;
    return v;
}
void gsl_vector_complex_free(gsl_vector_complex *v) {
    if (!v) return;
    free(v->data);
    free(v);
}
gsl_complex gsl_vector_complex_get(const gsl_vector_complex *v, const size_t i) {
    gsl_complex z;
    z.dat[0] = v->data[2 * i * v->stride];
    z.dat[1] = v->data[2 * i * v->stride + 1];
    return z;
}
gsl_matrix_complex *gsl_matrix_complex_alloc(const size_t n1, const size_t n2) {
    gsl_matrix_complex *m = (gsl_matrix_complex *)calloc(1, sizeof(*m));
    m->size1 = n1;
    m->size2 = n2;
    m->tda = n2;
    m->data = (double *)calloc(2 * n1 * n2, sizeof(double));
    m->owner = 1;
    return m;
}
void gsl_matrix_complex_free(gsl_matrix_complex *m) {
    if (!m) return;
    free(m->data);
    free(m);
}
gsl_vector_complex_view gsl_matrix_complex_column(gsl_matrix_complex *m, const size_t j) {
    gsl_vector_complex_view v;
    memset(&v, 0, sizeof(v));
    v.vector.size = m->size1;
    v.vector.stride = m->tda;
    v.vector.data = m->data + 2 * j;
    return v;
}
void gsl_matrix_complex_set(gsl_matrix_complex *m, const size_t i, const size_t j, const gsl_complex x) {
    m->data[2 * (i * m->tda + j)] = x.dat[0];
    m->data[2 * (i * m->tda + j) + 1] = x.dat[1];
}
gsl_eigen_nonsymmv_workspace *gsl_eigen_nonsymmv_alloc(const size_t n) {
    (void)n;
    return (gsl_eigen_nonsymmv_workspace *)calloc(1, sizeof(gsl_eigen_nonsymmv_workspace));
}
void gsl_eigen_nonsymmv_free(gsl_eigen_nonsymmv_workspace *w) { free(w); }

/* Cyclic Jacobi rotations (Golub & Van Loan, sec. 8.5) on a symmetric 3x3. */
int gsl_eigen_nonsymmv(gsl_matrix *A, gsl_vector_complex *eval, gsl_matrix_complex *evec,
                       gsl_eigen_nonsymmv_workspace *w) {
    double a[3][3], v[3][3];
    int i, j, p, q, sweep;
    (void)w;
    if (A->size1 != 3 || A->size2 != 3) shim_abort("gsl_eigen_nonsymmv (n != 3)");
    for (i = 0; i < 3; i++)
        for (j = 0; j < 3; j++) {
            a[i][j] = 0.5 * (A->data[i * A->tda + j] + A->data[j * A->tda + i]);
            v[i][j] = i == j;
        }
    for (sweep = 0; sweep < 64; sweep++) {
        double off = fabs(a[0][1]) + fabs(a[0][2]) + fabs(a[1][2]);
        if (off == 0.0) break;
        for (p = 0; p < 2; p++)
            for (q = p + 1; q < 3; q++) {
                double th, t, c, s;
                int k;
                if (a[p][q] == 0.0) continue;
                th = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                c = 1.0 / sqrt(t * t + 1.0);
                s = t * c;
                for (k = 0; k < 3; k++) {
                    double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
                for (k = 0; k < 3; k++) {
                    double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
                for (k = 0; k < 3; k++) {
                    double vkp = v[k][p], vkq = v[k][q];
                    v[k][p] = c * vkp - s * vkq;
                    v[k][q] = s * vkp + c * vkq;
                }
            }
    }
    for (i = 0; i < 3; i++) {
        eval->data[2 * i] = a[i][i];
        eval->data[2 * i + 1] = 0.0;
        for (j = 0; j < 3; j++) {
            evec->data[2 * (j * evec->tda + i)] = v[j][i];
            evec->data[2 * (j * evec->tda + i) + 1] = 0.0;
        }
    }
    return GSL_SUCCESS;
}

int gsl_eigen_nonsymmv_sort(gsl_vector_complex *eval, gsl_matrix_complex *evec, gsl_eigen_sort_t sort_type) {
    /* descending |value|; vectors follow */
    int i, j, k;
    (void)sort_type;
    for (i = 0; i < 2; i++)
        for (j = i + 1; j < 3; j++)
            if (fabs(eval->data[2 * j]) > fabs(eval->data[2 * i])) {
                double t = eval->data[2 * i];
                eval->data[2 * i] = eval->data[2 * j];
                eval->data[2 * j] = t;
                for (k = 0; k < 3; k++) {
                    double u = evec->data[2 * (k * evec->tda + i)];
                    evec->data[2 * (k * evec->tda + i)] = evec->data[2 * (k * evec->tda + j)];
                    evec->data[2 * (k * evec->tda + j)] = u;
                }
            }
    return GSL_SUCCESS;
}

/* ---------------- unreachable on the oracle paths ---------------- */
gsl_eigen_hermv_workspace *gsl_eigen_hermv_alloc(const size_t n) { (void)n; shim_abort("gsl_eigen_hermv_alloc"); return NULL; }
void gsl_eigen_hermv_free(gsl_eigen_hermv_workspace *w) { (void)w; shim_abort("gsl_eigen_hermv_free"); }
int gsl_eigen_hermv(gsl_matrix_complex *A, gsl_vector *eval, gsl_matrix_complex *evec, gsl_eigen_hermv_workspace *w) {
    (void)A; (void)eval; (void)evec; (void)w;
    shim_abort("gsl_eigen_hermv");
    return 0;
}
int gsl_eigen_hermv_sort(gsl_vector *eval, gsl_matrix_complex *evec, gsl_eigen_sort_t sort_type) {
    (void)eval; (void)evec; (void)sort_type;
    shim_abort("gsl_eigen_hermv_sort");
    return 0;
}

/* spglib (symmetry analysis; off the oracle paths) */
void spg_free_dataset(void *d) { (void)d; shim_abort("spg_free_dataset"); }
void *spg_get_dataset(void) { shim_abort("spg_get_dataset"); return NULL; }
int spg_get_international(void) { shim_abort("spg_get_international"); return 0; }
int spg_get_symmetry_from_database(void) { shim_abort("spg_get_symmetry_from_database"); return 0; }
int spg_standardize_cell(void) { shim_abort("spg_standardize_cell"); return 0; }
