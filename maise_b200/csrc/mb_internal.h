/*
 * mb_internal.h -- data structures shared by the C host code and the CUDA
 * kernels of libmaise_b200.
 */
#ifndef MB_INTERNAL_H
#define MB_INTERNAL_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MB_MAXSPC 3    /* the reference sizes its pair-parameter table W[9] for 3 species */
#define MB_NPAIR 9     /* pair index s0*s0 + s1*s1 (src/nprs.c:141-149) */
#define MB_MAXG2 32
#define MB_MAXE 10     /* eta values of G4 (one basis row holds at most 10) */
#define MB_MAXZ 10
#define MB_MAXL 10
#define MB_MAXZL 32
#define MB_MAXG4 160
#define MB_MAXD 1024
#define MB_MAXH 32     /* hidden-layer width */

/* Device-resident descriptor and network parameters of one model.  The
 * forward (energy) terms use the species-pair mixed parameters W[s0^2+s1^2]
 * and the derivative terms the species-0 block P, as the reference does
 * (src/nprs.c:504-566 vs 567-770). */
typedef struct {
    int nspc, D, ng2, ng4, ne, nz, nlam, nzl, h1, h2;
    int ind2[4], ind4[20];
    /* forward parameters per pair index p = s0*s0+s1*s1 */
    double f_rc2[MB_NPAIR], f_rc4[MB_NPAIR], f_rc4sq[MB_NPAIR];
    /* the smallest double t with sqrt(t) >= f_rc4: s < t exactly when
     * sqrt(s) < f_rc4, the reference's test of a triplet's j-k distance
     * (src/nprs.c:536) without a square root */
    double f_rc4thr[MB_NPAIR];
    double f_eta2[MB_NPAIR][MB_MAXG2], f_rs[MB_NPAIR][MB_MAXG2];
    double f_eta4[MB_NPAIR][MB_MAXE];
    /* derivative parameters (species-0 block) */
    double d_rc2, d_rc4, d_rc4sq;
    double d_eta2[MB_MAXG2], d_rs[MB_MAXG2], d_eta4[MB_MAXE];
    /* angular parameters (species-0 block) */
    double zeta[MB_MAXZ], lam[MB_MAXL], powz[MB_MAXZ];
    int zeta_int;            /* all zeta are integers in [1,64]: powers by squaring */
    int zeta_std;            /* zeta = {1, 2, 4, 16} exactly (the reference bases) */
    int zbits[MB_MAXZ];      /* bit pattern of zeta   (integer case) */
    int zm1bits[MB_MAXZ];    /* bit pattern of zeta-1 (integer case) */
    /* G4 feature f -> (eta index, zeta*nlam+lambda index) */
    int g4_e[MB_MAXG4], g4_zl[MB_MAXG4];
    /* UREP radii by species (mindist of the species' atomic number) */
    double rm[MB_MAXSPC];
    /* offsets (in doubles) of each species' network in the weight buffer */
    int w_off[MB_MAXSPC];
} mb_params;

/* Per-species network layout inside the weight buffer, starting at w_off[s]:
 *   off[D]      input shift Rmin*DR (src/nmlp.c:380)
 *   W0[h1][D]   first layer, input scaling folded in (src/nutl.c:621-630)
 *   b0[h1]
 *   W1[h2][h1], b1[h2]
 *   W2[h2], b2[1]
 */
#define MB_NET_SIZE(D, h1, h2) ((D) + (h1) * (D) + (h1) + (h2) * (h1) + (h2) + (h2) + 1)

/* Host copy of a parsed model. */
typedef struct {
    int nspc, spcz[MB_MAXSPC];
    int nl, nu[4], nw;
    mb_params P;
    double rc_list;          /* neighbour-list cutoff */
    double *weights;         /* host copy of the weight buffer */
    size_t weights_len;
    double mass[MB_MAXSPC];  /* amu * 103.6427 (src/cmod.c:1130) */
} mb_model;

int mb_model_load(const char *path, mb_model *m, char *err, size_t errlen);
void mb_model_free(mb_model *m);

/* Lattice data passed to kernels by value. */
typedef struct {
    double L[9];   /* rows = lattice vectors */
    double R[9];   /* reciprocal rows (no 2 pi), src/cell.c:432-443 */
    int ND;        /* periodic directions */
    int Nq[3];     /* image range ceil(Rc |R_q|) per periodic direction */
    int M[3];      /* cell-list bins per direction (0: brute force) */
} mb_cell;

/* leg-table path of the descriptor pass: one row per neighbour-list entry,
 * exp(-eta_e r^2) for e < 8, fc(r), fc'(r)/r */
#define MB_LEG_STRIDE 10
#define MB_LEG_MAX_ATOMS (1 << 17) /* atom index in 17 bits of an entry key */
#define MB_LEG_MAX_IMAGE 15        /* |image| per axis in 5 bits of an entry key */
#define MB_LEG_MAX_CAP 128         /* neighbour capacity the leg kernels handle */

/* status bits written by kernels */
#define MB_ST_NBR_OVERFLOW 1   /* an atom reached NM neighbours */
#define MB_ST_CAP_OVERFLOW 2   /* more neighbours than device capacity */
#define MB_ST_WRAP 4           /* non-finite position or unbounded wrap */

/* kernel modes */
#define MB_MODE_DESCRIPTORS 0
#define MB_MODE_ENERGY 1
#define MB_MODE_EFS 2
#define MB_MODE_VJP 3

/* multi-CTA reductions (k_finalize, k_nvt_thermostat): at most this many CTAs */
#define MB_RED_MAXB 64

/* Device working set of one handle (all pointers are device memory). */
typedef struct {
    int capN, capNB, capCells;
    double *X;        /* [3N] positions */
    double *V;        /* [3N] velocities (MD) */
    int *spc;         /* [N] species */
    int *nn;          /* [N] neighbour counts */
    int *nj;          /* [N*capNB] neighbour atoms */
    double *nd;       /* [N*capNB*4] dx,dy,dz,r */
    double *F;        /* [3N] forces */
    double *EA;       /* [N] MLP energies per atom */
    double *EU;       /* [N] repulsion energy per atom */
    double *vir;      /* [N*6] virial per central atom */
    double *G;        /* [N*D] descriptors or external weights (VJP) */
    int *cell_of;     /* [N] */
    int *cell_cnt;    /* [capCells] */
    int *cell_start;  /* [capCells+1] */
    int *cell_atoms;  /* [N] */
    double *out;      /* [16] E, H, U[6], K, xi, ... */
    double *part;     /* [2*MB_RED_MAXB*8] per-CTA partial sums of the reductions; NULL: one CTA */
    unsigned *ticket; /* [2] CTAs finished, per reduction kernel (reset by the last one) */
    double *trace;    /* [2*steps] H and K per MD step */
    int capTrace;
    int *status;      /* [4]: flags, max neighbour count */
    unsigned long long *counters; /* [2]: pairs and triplets seen by the descriptor kernel */
    mb_params *params;
    double *weights;
    /* leg tables (see mb_kernels.cu, k_legs): with legs_on the list kernels
     * also write each entry's key (atom << 15 | image, 5 bits per axis),
     * k_legs sorts every atom's list by species (nso[4N]: species starts
     * and the count) and fills leg[N*capNB*MB_LEG_STRIDE] with each entry's
     * exp(-eta_e r^2), fc(r) and fc'(r)/r; NULL where not allocated */
    unsigned *nk;
    double *leg;
    int *nso;
    /* triplet lists of the leg path (k_trip): trip[N*tcap] entries
     * {a | b << 8, j-k leg row} per atom, tboff[8N] the species blocks'
     * starts and the end; tcap = capNB (capNB - 1) / 2 bounds any list */
    void *trip;
    int *tboff;
    int tcap;
    void *lhash;      /* [N*256] uint2 (key, slot) per atom: the hash of its list (k_legs) */
    int legs_on;
    /* optional CUDA-event timing of the descriptor kernel */
    int ev_on, ev_n, ev_cap;
    void *ev_pool;    /* cudaEvent_t[2*ev_cap] */
    /* optional per-MD-step timing with an L2 flush between steps */
    int st_on, st_n, st_cap;
    void *st_pool;    /* cudaEvent_t[2*st_cap] */
    void *flush;
    size_t flush_bytes;
    /* kernel-shape autotuner cache (see mb_kernels.cu) */
#define MB_TUNE_SLOTS 32
    int tune_n, tune_fixed, last_shape;
    int tune_key[MB_TUNE_SLOTS], tune_val[MB_TUNE_SLOTS];
} mb_dev;

/* Launchers (mb_kernels.cu).  All enqueue on `stream`; return 0 or a CUDA
 * error code.  Counts of launched kernels are added to *launches. */
int mbk_wrap(mb_dev *d, int N, const mb_cell *c, void *stream, long *launches);
int mbk_nlist(mb_dev *d, int N, int NM, const mb_cell *c, double rc, void *stream, long *launches);
int mbk_descriptor_pass(mb_dev *d, const mb_model *m, int N, int mode, double urep, int need_nb_max, int nb_max,
                        void *stream, long *launches);
int mbk_finalize(mb_dev *d, int N, int mode, double pV, void *stream, long *launches);
int mbk_jvp(mb_dev *d, const mb_model *m, int N, const double *dx, const double *eps, double *dG, void *stream,
            long *launches);
/* thermostat and integrator, then JAR on the moved atoms (cell c; none when c->ND <= 0) */
int mbk_nvt_update(mb_dev *d, const mb_model *m, int N, double dt, double tau, double T, const mb_cell *c,
                   void *stream, long *launches);
int mbk_set_out(mb_dev *d, int idx, double v, void *stream);
void mbk_record(void *event, void *stream);
int mbk_shape_ready(const mb_dev *d, int N, int mode);
int mbk_legs_model(const mb_model *m);
int mbk_legs_usable(const mb_dev *d, const mb_model *m, int N, const mb_cell *c);
int mbk_shape_dims(int legs, int shape, int *wpa, int *apb);
int mbk_graph_cell_nodes(void *graph, void **nodes, int *rows, int cap);
int mbk_graph_set_cell(void *exec, void *const *nodes, const int *rows, int count, const mb_cell *c, double pV);
size_t mbk_efs_smem(const mb_model *m, int capNB, int shape);

#ifdef __cplusplus
}
#endif
#endif
