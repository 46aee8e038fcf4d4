/*
 * oracle.c -- CPU restatement of MAISE's neural-network potential path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product
 * path: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg may load the library built from it.  Nothing in maise_b200/ links or
 * calls it.
 *
 * It restates, in plain FP64 C, what the reference computes for one
 * structure (file:line refer to the maise 3.0.00 sources):
 *   - model file parsing and the input-normalisation fold
 *       (src/util.c:1233-1335 READ_MODEL, src/nutl.c:502-633 READ_ANN,
 *        src/nmlp.c:591-608 V2W)
 *   - basis parsing, B2A unit scaling and species-pair mixing
 *       (src/nprs.c:75-257 Build_PRS)
 *   - wrap into the cell and the brute-force periodic neighbour list
 *       (src/cell.c:432-508 Relative/Real/JAR, src/cell.c:82-185 LIST)
 *   - G2/G4 descriptors, their Cartesian derivatives dG_j/dx_i and strain
 *       derivatives (src/nprs.c:445-773 PRS_BP)
 *   - per-species MLP energy and the force/virial contraction
 *       (src/nmlp.c:367-488 ENE_ANN/FRC_ANN)
 *   - short-range repulsion (src/cmod.c:61-126 CELL_UREP), noise zeroing and
 *       enthalpy (src/cmod.c:128-191 CELL_ENE/CELL_FRC)
 *
 * Unlike the product it follows the reference's formulation: the full
 * per-neighbour derivative blocks Fn[i][j][l][3] and Sn[i][l][6] are
 * materialised and contracted afterwards, exactly the data the reference
 * writes to its parse files (src/nprs.c:380-442).  Parity against the
 * reference itself is pinned by tests against the golden e-files of
 * test/parse/ref and against the reference sources compiled under
 * oracle/_ref.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MAXSPC 3     /* the reference sizes W[9] for at most 3 species (src/nmod.c, src/cmod.c:1187) */
#define ORC_NPAR 10      /* parameter values per basis row (src/nprs.c:87) */

static const double ORC_PI = 3.1415926535897932384626433832795;   /* src/util.c:3 */
static const double ORC_EV2GPA = 160.2176565;                      /* src/util.c:8 */

/* Minimum interatomic distances in Angstrom by atomic number, the UREP radii
 * (src/util.c:13).  Physical data that must match the reference exactly. */
static const double orc_mindist[96] = {
    0.0, 1.0, 1.0, 1.040, 0.773, 0.584, 0.499, 1.0, 1.0, 1.0, 1.0, 1.266, 1.114, 1.0, 1.0, 1.0,
    1.0, 1.0, 1.0, 1.610, 1.366, 1.123, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 0.895, 1.0, 1.0,
    1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 0.979, 1.030,
    1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0,
    1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 0.984, 1.0,
    1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0};

/* one basis block: function table and scaled parameter rows */
typedef struct {
    int nsym;
    int gf[512][8];          /* type, Rc, Rs, eta2, eta4, k, zeta, lambda indices */
    int gt[7];               /* number of values in each parameter row */
    double gp[7][ORC_NPAR];  /* Rc, Rs, eta2, eta4, k, zeta, lambda */
} orc_block;

typedef struct {
    int nspc, spcz[ORC_MAXSPC];
    int nl, nu[4], nw, D;
    double *Rmin[ORC_MAXSPC], *DR[ORC_MAXSPC]; /* folded: Rmin/DR (src/nutl.c:627-629) */
    double *W[ORC_MAXSPC][3];                  /* W[s][k][m*nu[k]+n], W0 folded by DR */
    double *B[ORC_MAXSPC][3];
    orc_block blk[9];  /* indexed by s0*s0+s1*s1 as in the reference W[9] */
    int ng2, ng4;
    double rc_list;    /* neighbour-list cutoff (src/nprs.c:456-462) */
} orc_model;

/* ------------------------------------------------------------------ */
/* model file parsing                                                  */
/* ------------------------------------------------------------------ */

static int orc_find(FILE *f, const char *key, int n, char *line) {
    while (fgets(line, 400, f))
        if (strncmp(line, key, n) == 0) return 1;
    return 0;
}

/* version check: "|  maise version | maise.X.Y.Z |" -> X*1000+Y*100+Z (src/util.c:1948-1996) */
static int orc_version(const char *path) {
    FILE *f = fopen(path, "r");
    char line[400], tok[200];
    int v[3] = {0, 0, 0}, i = 0;
    if (!f) return -2;
    if (!fgets(line, 400, f) || !fgets(line, 400, f)) { fclose(f); return -1; }
    if (sscanf(line + 2, "%199s", tok) != 1 || strncmp(tok, "neural", 6) != 0) { fclose(f); return -1; }
    if (!orc_find(f, "|  maise version", 16, line)) { fclose(f); return -1; }
    fclose(f);
    if (sscanf(line, "|  maise version | %199s |", tok) != 1) return -1;
    /* after "maise." come dot-separated integer fields */
    {
        char *p = tok + 6;
        while (i < 3 && *p) {
            v[i++] = atoi(p);
            while (*p && *p != '.') p++;
            if (*p == '.') p++;
        }
    }
    return v[0] * 1000 + v[1] * 100 + v[2];
}

/* Parse the basis section that follows the "  B2A" line (src/nprs.c:141-256). */
static int orc_parse_basis(orc_model *M, const char *path, char *err) {
    FILE *f = fopen(path, "r");
    char line[400], name[64];
    int s, n, q, nsym = -1;
    long b2a_pos;
    if (!f) { sprintf(err, "cannot open %s", path); return -1; }
    /* NSYM = lines between the 4 header lines and " Rc  ", minus one blank (src/util.c:1310-1318) */
    if (!orc_find(f, "  B2A", 5, line)) { fclose(f); sprintf(err, "no B2A section"); return -1; }
    b2a_pos = ftell(f);
    for (q = 0; q < 4; q++) fgets(line, 400, f);
    while (fgets(line, 400, f)) {
        if (strncmp(line, " Rc  ", 5) == 0) break;
        nsym++;
    }
    if (nsym <= 0 || nsym > 512) { fclose(f); sprintf(err, "bad NSYM %d", nsym); return -1; }
    fseek(f, b2a_pos, SEEK_SET);
    for (s = 0; s < M->nspc; s++) {
        orc_block *B = &M->blk[2 * s * s];
        double a, r;
        if (!fgets(line, 400, f) || sscanf(line, "%lf %lf", &a, &r) != 2) {
            fclose(f); sprintf(err, "bad B2A scale line"); return -1;
        }
        for (q = 0; q < 3; q++) fgets(line, 400, f);
        B->nsym = nsym;
        for (n = 0; n < nsym; n++) {
            int idx;
            fgets(line, 400, f);
            if (sscanf(line, "%d %d %d %d %d %d %d %d %d", &idx, &B->gf[n][0], &B->gf[n][1], &B->gf[n][2],
                       &B->gf[n][3], &B->gf[n][4], &B->gf[n][5], &B->gf[n][6], &B->gf[n][7]) != 9) {
                fclose(f); sprintf(err, "bad basis function line %d", n); return -1;
            }
        }
        fgets(line, 400, f);
        for (n = 0; n < 7; n++) {
            double *g = B->gp[n];
            for (q = 0; q < ORC_NPAR; q++) g[q] = 0.0;
            fgets(line, 400, f);
            if (sscanf(line, "%63s %d %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf", name, &B->gt[n], &g[0], &g[1],
                       &g[2], &g[3], &g[4], &g[5], &g[6], &g[7], &g[8], &g[9]) < 3) {
                fclose(f); sprintf(err, "bad parameter row %d", n); return -1;
            }
        }
        /* B2A scaling: lengths times a*r, exponents divided by (a*r)^2 (src/nprs.c:183-189) */
        for (n = 0; n < 2; n++)
            for (q = 0; q < ORC_NPAR; q++) B->gp[n][q] *= a * r;
        for (n = 2; n < 4; n++)
            for (q = 0; q < ORC_NPAR; q++) B->gp[n][q] /= a * a * r * r;
        fgets(line, 400, f);
        /* a missing further block means: reuse the first block (src/nprs.c:223-231) */
        if (s < M->nspc - 1 && fgets(line, 400, f) == NULL) {
            fseek(f, b2a_pos, SEEK_SET);
        }
    }
    fclose(f);
    /* off-diagonal pair mixing (src/nprs.c:233-252) */
    for (s = 0; s < M->nspc; s++)
        for (q = 0; q < M->nspc; q++)
            if (s != q) {
                orc_block *A = &M->blk[2 * s * s], *C = &M->blk[2 * q * q], *X = &M->blk[s * s + q * q];
                int i;
                *X = M->blk[0];
                for (n = 0; n < 2; n++)
                    for (i = 0; i < ORC_NPAR; i++) X->gp[n][i] = 0.5 * (A->gp[n][i] + C->gp[n][i]);
                for (n = 2; n < 4; n++)
                    for (i = 0; i < ORC_NPAR; i++)
                        X->gp[n][i] = pow(0.5 * (pow(A->gp[n][i], -0.5) + pow(C->gp[n][i], -0.5)), -2.0);
            }
    /* counts of G2/G4 functions; G2 functions must come first */
    M->ng2 = M->ng4 = 0;
    for (n = 0; n < nsym; n++) {
        int t = M->blk[0].gf[n][0];
        if (t == 2) {
            if (M->ng4) { sprintf(err, "G2 after G4 in basis"); return -1; }
            M->ng2++;
        } else if (t == 4) {
            M->ng4++;
        } else {
            sprintf(err, "unsupported basis function type %d", t); return -1;
        }
    }
    {
        int c = M->nspc * (M->nspc + 1) / 2;
        if (M->ng2 * M->nspc + M->ng4 * c != M->D) {
            sprintf(err, "NCMP %d inconsistent with basis (%d)", M->D, M->ng2 * M->nspc + M->ng4 * c);
            return -1;
        }
    }
    /* neighbour-list cutoff: the smallest Rc of any function in any species block (src/nprs.c:455-462) */
    M->rc_list = M->blk[0].gp[0][0];
    for (s = 0; s < M->nspc; s++)
        for (n = 0; n < nsym; n++) {
            double rc = M->blk[2 * s * s].gp[0][M->blk[0].gf[n][1]];
            if (M->rc_list > rc) M->rc_list = rc;
        }
    return 0;
}

void orc_model_free(orc_model *M) {
    int s, k;
    if (!M) return;
    for (s = 0; s < ORC_MAXSPC; s++) {
        free(M->Rmin[s]);
        free(M->DR[s]);
        for (k = 0; k < 3; k++) { free(M->W[s][k]); free(M->B[s][k]); }
    }
    free(M);
}

orc_model *orc_model_load(const char *path, char *err) {
    orc_model *M;
    FILE *f;
    char line[400];
    int s, k, n, m, i;
    double *V;
    if (orc_version(path) < 2400) { sprintf(err, "model missing or older than format 2.4.00"); return NULL; }
    f = fopen(path, "r");
    if (!f) { sprintf(err, "cannot open %s", path); return NULL; }
    M = (orc_model *)calloc(1, sizeof(orc_model));
    if (!orc_find(f, "|  number of species    |", 25, line)) goto bad;
    sscanf(line + 26, "%d", &M->nspc);
    if (M->nspc < 1 || M->nspc > ORC_MAXSPC) goto bad;
    if (!orc_find(f, "|  species types        |", 25, line)) goto bad;
    {
        char *p = line + 26;
        int used;
        for (s = 0; s < M->nspc; s++) {
            if (sscanf(p, "%d%n", &M->spcz[s], &used) != 1) goto bad;
            p += used;
        }
    }
    if (!orc_find(f, "|  number of layers     |", 25, line)) goto bad;
    sscanf(line + 26, "%d", &M->nl);
    if (M->nl != 4) { sprintf(err, "only 2 hidden layers are supported (NL=%d)", M->nl); fclose(f); orc_model_free(M); return NULL; }
    if (!orc_find(f, "|  architecture         |", 25, line)) goto bad;
    {
        char *p = line + 26;
        int used;
        for (k = 0; k < 4; k++) {
            if (sscanf(p, "%d%n", &M->nu[k], &used) != 1) goto bad;
            p += used;
        }
    }
    M->D = M->nu[0];
    if (!orc_find(f, "|  number of weights    |", 25, line)) goto bad;
    sscanf(line + 26, "%d", &M->nw);
    if (!orc_find(f, "        minimum          ", 25, line)) goto bad;
    for (s = 0; s < M->nspc; s++) {
        double mx;
        M->Rmin[s] = (double *)malloc(sizeof(double) * M->D);
        M->DR[s] = (double *)malloc(sizeof(double) * M->D);
        for (n = 0; n < M->D; n++)
            if (fscanf(f, "%lf %lf %lf", &M->Rmin[s][n], &mx, &M->DR[s][n]) != 3) goto bad;
    }
    /* skip to the weights block */
    if (!orc_find(f, "|                        neural network weights", 40, line)) goto bad;
    fgets(line, 400, f);
    V = (double *)malloc(sizeof(double) * M->nw);
    for (i = 0; i < M->nw; i++)
        if (fscanf(f, "%lf", &V[i]) != 1) { free(V); goto bad; }
    fclose(f);
    f = NULL;
    /* V2W order: per species, all biases first then all weights (src/nmlp.c:591-608) */
    i = 0;
    for (s = 0; s < M->nspc; s++) {
        for (k = 0; k < 3; k++) {
            M->B[s][k] = (double *)malloc(sizeof(double) * M->nu[k + 1]);
            M->W[s][k] = (double *)malloc(sizeof(double) * M->nu[k + 1] * M->nu[k]);
        }
        for (k = 0; k < 3; k++)
            for (m = 0; m < M->nu[k + 1]; m++) M->B[s][k][m] = V[i++];
        for (k = 0; k < 3; k++)
            for (m = 0; m < M->nu[k + 1]; m++)
                for (n = 0; n < M->nu[k]; n++) M->W[s][k][m * M->nu[k] + n] = V[i++];
    }
    free(V);
    if (i != M->nw) { sprintf(err, "weight count mismatch"); orc_model_free(M); return NULL; }
    /* fold the input scaling into the first layer (src/nutl.c:621-630) */
    for (s = 0; s < M->nspc; s++) {
        for (m = 0; m < M->nu[1]; m++)
            for (n = 0; n < M->nu[0]; n++) M->W[s][0][m * M->nu[0] + n] *= M->DR[s][n];
        for (n = 0; n < M->nu[0]; n++) M->Rmin[s][n] /= M->DR[s][n];
    }
    if (orc_parse_basis(M, path, err)) { orc_model_free(M); return NULL; }
    return M;
bad:
    if (f) fclose(f);
    sprintf(err, "malformed model file %s", path);
    orc_model_free(M);
    return NULL;
}

int orc_model_info(const orc_model *M, int *nspc, int *D, int *spcz, double *rc_list, int *ng2, int *ng4) {
    int s;
    *nspc = M->nspc;
    *D = M->D;
    for (s = 0; s < M->nspc; s++) spcz[s] = M->spcz[s];
    *rc_list = M->rc_list;
    *ng2 = M->ng2;
    *ng4 = M->ng4;
    return 0;
}

/* ------------------------------------------------------------------ */
/* geometry                                                            */
/* ------------------------------------------------------------------ */

/* reciprocal vectors without 2*pi (src/cell.c:432-443) */
static void orc_reciprocal(const double L[3][3], double R[3][3]) {
    double t;
    int i, q;
    R[2][0] = L[0][1] * L[1][2] - L[0][2] * L[1][1];
    R[2][1] = L[0][2] * L[1][0] - L[0][0] * L[1][2];
    R[2][2] = L[0][0] * L[1][1] - L[0][1] * L[1][0];
    R[0][0] = L[1][1] * L[2][2] - L[1][2] * L[2][1];
    R[0][1] = L[1][2] * L[2][0] - L[1][0] * L[2][2];
    R[0][2] = L[1][0] * L[2][1] - L[1][1] * L[2][0];
    R[1][0] = L[2][1] * L[0][2] - L[2][2] * L[0][1];
    R[1][1] = L[2][2] * L[0][0] - L[2][0] * L[0][2];
    R[1][2] = L[2][0] * L[0][1] - L[2][1] * L[0][0];
    t = 1.0 / (L[0][0] * L[1][1] * L[2][2] + L[0][1] * L[1][2] * L[2][0] + L[0][2] * L[1][0] * L[2][1] -
               L[0][0] * L[1][2] * L[2][1] - L[0][1] * L[1][0] * L[2][2] - L[0][2] * L[1][1] * L[2][0]);
    for (i = 0; i < 3; i++)
        for (q = 0; q < 3; q++) R[i][q] *= t;
}

/* wrap into [0,1) in fractional coordinates and back (src/cell.c:445-508) */
static void orc_wrap(int N, double *X, const double L[3][3]) {
    double R[3][3], x[3];
    int i, q, j;
    orc_reciprocal(L, R);
    for (i = 0; i < N; i++) {
        for (q = 0; q < 3; q++) {
            x[q] = 0.0;
            for (j = 0; j < 3; j++) x[q] += X[3 * i + j] * R[q][j];
        }
        for (q = 0; q < 3; q++) {
            while (x[q] < 0.0) x[q] += 1.0;
            while (x[q] >= 1.0) x[q] -= 1.0;
        }
        for (q = 0; q < 3; q++) {
            double c = 0.0;
            for (j = 0; j < 3; j++) c += x[j] * L[j][q];
            X[3 * i + q] = c;
        }
    }
}

double orc_cell_volume(const double L[3][3]) {
    /* src/cutl.c:178-188 for periodic cells */
    double V = L[0][0] * L[1][1] * L[2][2] + L[0][2] * L[1][0] * L[2][1] + L[0][1] * L[1][2] * L[2][0] -
               L[0][0] * L[1][2] * L[2][1] - L[0][1] * L[1][0] * L[2][2] - L[0][2] * L[1][1] * L[2][0];
    return fabs(V);
}

/* Neighbour list: every atom j and periodic image within Rc of atom i,
 * excluding i's own zero image (src/cell.c:82-185).  The shift vector and
 * distance are formed with the same operations as the reference so that the
 * strict test r^2 < Rc^2 selects the same set.  Returns -1 if an atom
 * reaches NM neighbours (the reference aborts there, src/cell.c:134-142). */
typedef struct {
    int N, NM;
    int *nn;      /* [N] */
    int *j;       /* [N*NM] neighbour atom */
    int *ic;      /* [N*NM*3] image indices */
    double *d;    /* [N*NM*3] DX = X_j + S - X_i */
    double *r;    /* [N*NM] */
} orc_list;

static void orc_list_free(orc_list *T) {
    free(T->nn); free(T->j); free(T->ic); free(T->d); free(T->r);
}

static int orc_build_list(int N, int NM, int ND, const double *X, const double L[3][3], double Rc, orc_list *T) {
    double R[3][3], RC = Rc * Rc;
    int Nq[3] = {0, 0, 0}, i, q;
    T->N = N; T->NM = NM;
    T->nn = (int *)calloc(N, sizeof(int));
    T->j = (int *)calloc((size_t)N * NM, sizeof(int));
    T->ic = (int *)calloc((size_t)N * NM * 3, sizeof(int));
    T->d = (double *)calloc((size_t)N * NM * 3, sizeof(double));
    T->r = (double *)calloc((size_t)N * NM, sizeof(double));
    orc_reciprocal(L, R);
    for (q = 0; q < ND; q++) Nq[q] = (int)ceil(Rc * sqrt(R[q][0] * R[q][0] + R[q][1] * R[q][1] + R[q][2] * R[q][2]));
    for (i = 0; i < N; i++) {
        int c = 0, j, a, b, e, k;
        double r2s[4096];
        double *rr = NM <= 4096 ? r2s : (double *)malloc(sizeof(double) * NM);
        for (j = 0; j < N; j++)
            for (a = -Nq[0]; a <= Nq[0]; a++)
                for (b = -Nq[1]; b <= Nq[1]; b++)
                    for (e = -Nq[2]; e <= Nq[2]; e++) {
                        double r = 0.0, dv[3];
                        int ic[3] = {a, b, e};
                        if (i == j && a == 0 && b == 0 && e == 0) continue;
                        for (q = 0; q < 3; q++) {
                            double x = 0.0;
                            for (k = 0; k < 3; k++) x += (double)ic[k] * L[k][q];
                            x += X[3 * j + q] - X[3 * i + q];
                            dv[q] = x;
                            r += x * x;
                        }
                        if (r < RC) {
                            size_t o = (size_t)i * NM + c;
                            T->j[o] = j;
                            for (q = 0; q < 3; q++) { T->ic[3 * o + q] = ic[q]; T->d[3 * o + q] = dv[q]; }
                            rr[c] = r;
                            c++;
                            if (c == NM) { if (rr != r2s) free(rr); return -1; }
                        }
                    }
        /* nearest neighbour into slot 0 by the reference's swap sequence (src/cell.c:157-165) */
        for (j = 1; j < c; j++)
            if (rr[j] < rr[0]) {
                size_t o0 = (size_t)i * NM, oj = (size_t)i * NM + j;
                int ti = T->j[o0];
                double tr = rr[0];
                T->j[o0] = T->j[oj]; T->j[oj] = ti;
                for (q = 0; q < 3; q++) {
                    int t1 = T->ic[3 * o0 + q];
                    double t2 = T->d[3 * o0 + q];
                    T->ic[3 * o0 + q] = T->ic[3 * oj + q]; T->ic[3 * oj + q] = t1;
                    T->d[3 * o0 + q] = T->d[3 * oj + q]; T->d[3 * oj + q] = t2;
                }
                rr[0] = rr[j]; rr[j] = tr;
            }
        for (j = 0; j < c; j++) T->r[(size_t)i * NM + j] = sqrt(rr[j]);
        T->nn[i] = c;
        if (rr != r2s) free(rr);
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* descriptors                                                         */
/* ------------------------------------------------------------------ */

static double orc_fc(double Rc, double r) { return r > Rc ? 0.0 : 0.5 * (cos(ORC_PI * r / Rc) + 1.0); }
static double orc_dfc(double Rc, double r) { return r > Rc ? 0.0 : -0.5 * ORC_PI / Rc * sin(ORC_PI * r / Rc); }

/* species-resolved offsets of the G2 and G4 blocks (src/nprs.c:484-498) */
static void orc_offsets(const orc_model *M, int *ind2, int *ind4) {
    int a = M->ng2, b = M->ng4;
    memset(ind4, 0, sizeof(int) * 20);
    ind2[0] = 0; ind2[1] = a + b; ind2[2] = 2 * a + 3 * b; ind2[3] = 3 * a + 6 * b;
    ind4[0] = a; ind4[1] = 2 * a + b; ind4[2] = 2 * a + 2 * b; ind4[4] = 3 * a + 3 * b; ind4[8] = 3 * a + 4 * b;
    ind4[5] = 3 * a + 5 * b; ind4[9] = 4 * a + 6 * b; ind4[18] = 4 * a + 7 * b; ind4[10] = 4 * a + 8 * b;
    ind4[13] = 4 * a + 9 * b;
}

static double orc_dot(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* cos(angle j-i-k) and r_jk from the stored displacement vectors (src/cell.c:171-181) */
static void orc_angle(const orc_list *T, int i, int j, int k, double *c, double *rjk) {
    const double *dj = T->d + 3 * ((size_t)i * T->NM + j), *dk = T->d + 3 * ((size_t)i * T->NM + k);
    double a[3], r = 0.0;
    int q;
    for (q = 0; q < 3; q++) r += dj[q] * dk[q];
    *c = r / (T->r[(size_t)i * T->NM + j] * T->r[(size_t)i * T->NM + k]);
    for (q = 0; q < 3; q++) a[q] = dj[q] - dk[q];
    *rjk = sqrt(orc_dot(a, a));
}

/* Energy descriptors G[N][D] (src/nprs.c:500-566). */
static void orc_descriptors(const orc_model *M, const orc_list *T, const int *atmn, double *G) {
    const orc_block *P = &M->blk[0];
    int ind2[4], ind4[20], i, n, z, l;
    int ns = M->nspc, D = M->D, g2f = M->ng2;
    double powz[ORC_NPAR];
    orc_offsets(M, ind2, ind4);
    for (z = 0; z < P->gt[5]; z++) powz[z] = pow(2.0, 1.0 - P->gp[5][z]);
    memset(G, 0, sizeof(double) * (size_t)T->N * D);
    for (i = 0; i < T->N; i++) {
        int s0 = atmn[i], jj, k;
        double *Gi = G + (size_t)i * D;
        for (jj = 0; jj < T->nn[i]; jj++) {
            int s1 = atmn[T->j[(size_t)i * T->NM + jj]];
            const orc_block *W01 = &M->blk[s0 * s0 + s1 * s1];
            double rij = T->r[(size_t)i * T->NM + jj];
            double R01 = W01->gp[0][P->gf[0][1]];
            int ds1 = (s1 - s0 + ns) % ns, g2;
            if (!(rij < R01)) continue;
            for (n = 0, g2 = 0; n < P->nsym; n++)
                if (P->gf[n][0] == 2) {
                    double eta = W01->gp[2][P->gf[n][3]], rs = W01->gp[1][P->gf[n][2]];
                    Gi[g2 + ind2[ds1]] += orc_fc(R01, rij) * exp(-eta * pow(rij - rs, 2.0));
                    g2++;
                }
            if (!(g2f < D && rij < W01->gp[0][P->gf[g2f][1]])) continue;
            for (k = jj + 1; k < T->nn[i]; k++) {
                int s2 = atmn[T->j[(size_t)i * T->NM + k]];
                const orc_block *W02 = &M->blk[s0 * s0 + s2 * s2], *W12 = &M->blk[s1 * s1 + s2 * s2];
                double R02 = W02->gp[0][P->gf[g2f][1]], R12 = W12->gp[0][P->gf[g2f][1]];
                double rik = T->r[(size_t)i * T->NM + k], c, rjk, A, e[ORC_NPAR], lz[ORC_NPAR][ORC_NPAR];
                int ds2 = (s2 - s0 + ns) % ns, ds, g4;
                orc_angle(T, i, jj, k, &c, &rjk);
                if (!(rik < R02 && rjk < R12)) continue;
                A = 2.0 * orc_fc(R01, rij) * orc_fc(R02, rik) * orc_fc(R12, rjk);
                for (n = 0; n < P->gt[3]; n++)
                    e[n] = A * exp(-rij * rij * W01->gp[3][n] - rik * rik * W02->gp[3][n] - rjk * rjk * W12->gp[3][n]);
                for (z = 0; z < P->gt[5]; z++)
                    for (l = 0; l < P->gt[6]; l++) lz[z][l] = powz[z] * pow(1.0 + P->gp[6][l] * c, P->gp[5][z]);
                ds = ds1 * ds1 + ds2 * ds2;
                for (n = 0, g4 = 0; n < P->nsym; n++)
                    if (P->gf[n][0] == 4) {
                        Gi[g4 + ind4[ds]] += lz[P->gf[n][6]][P->gf[n][7]] * e[P->gf[n][4]];
                        g4++;
                    }
            }
        }
    }
}

/* Derivative blocks for atom i (src/nprs.c:567-770), restated:
 *   Fn[(slot*D + m)*3 + q] = dG_{m} of neighbour atom DNi[slot] w.r.t. x_i,
 *       slot < dnn: unique neighbour atoms in first-seen order;
 *       slot == dnn: dG_i/dx_i (self block)
 *   Sn[m*6 + c] = strain derivative of G_i (xx,yy,zz,xy,yz,zx)
 * All derivative terms use the species-0 parameter block, as the reference does. */
static void orc_derivatives(const orc_model *M, const orc_list *T, const int *atmn, int i, int *dnn_out, int *dni,
                            double *Fn, double *Sn) {
    const orc_block *P = &M->blk[0];
    int ind2[4], ind4[20], ns = M->nspc, D = M->D, g2f = M->ng2, n, z, l, q;
    int s0 = atmn[i], dnn = 0, jj, N = T->N, NM = T->NM;
    double powz[ORC_NPAR], Rc2 = P->gp[0][P->gf[0][1]], Rc4 = g2f < D ? P->gp[0][P->gf[g2f][1]] : 0.0;
    char *seen = (char *)calloc(N, 1);
    orc_offsets(M, ind2, ind4);
    for (z = 0; z < P->gt[5]; z++) powz[z] = pow(2.0, 1.0 - P->gp[5][z]);
    if (Fn) memset(Fn, 0, sizeof(double) * (size_t)(NM + 1) * D * 3);
    if (Sn) memset(Sn, 0, sizeof(double) * (size_t)D * 6);

    /* neighbour side: G_j depends on x_i through every image of i in j's list */
    if (Fn)
        for (jj = 0; jj < T->nn[i]; jj++) {
            int j = T->j[(size_t)i * NM + jj], s1 = atmn[j], ii;
            double *F = NULL;
            if (seen[j]) continue;
            seen[j] = 1;
            F = Fn + (size_t)dnn * D * 3;
            for (ii = 0; ii < T->nn[j]; ii++) {
                const double *dji;
                double rji;
                int g2, k;
                if (T->j[(size_t)j * NM + ii] != i) continue;
                dji = T->d + 3 * ((size_t)j * NM + ii);
                rji = T->r[(size_t)j * NM + ii];
                {
                    double fcij = orc_fc(Rc2, rji), dfcij = orc_dfc(Rc2, rji);
                    int ds1 = (s0 - s1 + ns) % ns;
                    for (n = 0, g2 = 0; n < P->nsym; n++)
                        if (P->gf[n][0] == 2) {
                            double eta = P->gp[2][P->gf[n][3]], rs = P->gp[1][P->gf[n][2]];
                            double t = exp(-eta * pow(rji - rs, 2.0)) * (-2.0 * eta * (rji - rs) * fcij + dfcij) / rji;
                            for (q = 0; q < 3; q++) F[(size_t)(g2 + ind2[ds1]) * 3 + q] += t * dji[q];
                            g2++;
                        }
                }
                if (!(g2f < D && rji < Rc4)) continue;
                for (k = 0; k < T->nn[j]; k++) {
                    const double *djk;
                    double c, rik, rjk, A0, a52, a53, a63, ijk, ex[ORC_NPAR];
                    int s2, ds, g4;
                    if (k == ii) continue;
                    orc_angle(T, j, ii, k, &c, &rik);
                    rjk = T->r[(size_t)j * NM + k];
                    if (!(rik < Rc4 && rjk < Rc4)) continue;
                    djk = T->d + 3 * ((size_t)j * NM + k);
                    A0 = orc_fc(Rc4, rji) * orc_fc(Rc4, rik);
                    for (n = 0; n < P->gt[3]; n++)
                        ex[n] = 2.0 * exp(-P->gp[3][n] * (rji * rji + rjk * rjk + rik * rik)) * orc_fc(Rc4, rjk);
                    s2 = atmn[T->j[(size_t)j * NM + k]];
                    ds = ((s0 - s1 + ns) % ns) * ((s0 - s1 + ns) % ns) + ((s2 - s1 + ns) % ns) * ((s2 - s1 + ns) % ns);
                    a52 = -c / rji;
                    a53 = orc_fc(Rc4, rik) * orc_dfc(Rc4, rji) / rji;
                    a63 = orc_fc(Rc4, rji) * orc_dfc(Rc4, rik) / rik;
                    ijk = 1.0 / rjk;
                    for (n = 0, g4 = 0; n < P->nsym; n++)
                        if (P->gf[n][0] == 4) {
                            double zz = P->gp[5][P->gf[n][6]], lam = P->gp[6][P->gf[n][7]], eta = P->gp[3][P->gf[n][4]];
                            double base = 1.0 + lam * c;
                            double A2 = powz[P->gf[n][6]] * A0 * lam * zz * pow(base, zz - 1.0) / rji;
                            double A3 = powz[P->gf[n][6]] * pow(base, zz);
                            double A4 = -2.0 * eta * A0;
                            double A5 = A2 * a52 + A3 * (a53 + A4), A6 = A3 * (a63 + A4), A7 = A2 * ijk;
                            double w = ex[P->gf[n][4]];
                            for (q = 0; q < 3; q++)
                                F[(size_t)(g4 + ind4[ds]) * 3 + q] += w * ((A5 + A6) * dji[q] + (A7 - A6) * djk[q]);
                            g4++;
                        }
                }
            }
            dni[dnn++] = j;
        }

    /* self side: dG_i/dx_i and the strain derivative */
    for (jj = 0; jj < T->nn[i]; jj++) {
        const double *dij = T->d + 3 * ((size_t)i * NM + jj);
        double rij = T->r[(size_t)i * NM + jj], dq[3], fcij = orc_fc(Rc2, rij), dfcij = orc_dfc(Rc2, rij);
        int s1 = atmn[T->j[(size_t)i * NM + jj]], ds1 = (s1 - s0 + ns) % ns, g2, k;
        double *Fs = Fn ? Fn + (size_t)dnn * D * 3 : NULL;
        for (q = 0; q < 3; q++) dq[q] = dij[(q + 1) % 3];
        for (n = 0, g2 = 0; n < P->nsym; n++)
            if (P->gf[n][0] == 2) {
                double eta = P->gp[2][P->gf[n][3]], rs = P->gp[1][P->gf[n][2]];
                double t = exp(-eta * pow(rij - rs, 2.0)) * (-2.0 * eta * (rij - rs) * fcij + dfcij) / rij;
                int m = g2 + ind2[ds1];
                if (Fs)
                    for (q = 0; q < 3; q++) Fs[(size_t)m * 3 + q] -= t * dij[q];
                if (Sn)
                    for (q = 0; q < 3; q++) {
                        Sn[(size_t)m * 6 + q] += t * dij[q] * dij[q];
                        Sn[(size_t)m * 6 + q + 3] += t * dij[q] * dq[q];
                    }
                g2++;
            }
        if (!(g2f < D && rij < Rc4)) continue;
        for (k = jj + 1; k < T->nn[i]; k++) {
            const double *dik = T->d + 3 * ((size_t)i * NM + k);
            double rik = T->r[(size_t)i * NM + k], c, rjk, dqk[3], ex[ORC_NPAR];
            double A0, T0, F0, F1, F2, a52, a62, a53, a63;
            int s2 = atmn[T->j[(size_t)i * NM + k]], ds2 = (s2 - s0 + ns) % ns, ds = ds1 * ds1 + ds2 * ds2, g4;
            orc_angle(T, i, jj, k, &c, &rjk);
            if (!(rjk < Rc4 && rik < Rc4)) continue;
            for (q = 0; q < 3; q++) dqk[q] = dik[(q + 1) % 3];
            A0 = orc_fc(Rc4, rij) * orc_fc(Rc4, rik);
            T0 = orc_fc(Rc4, rjk);
            F0 = orc_dfc(Rc4, rij) * orc_fc(Rc4, rik) * orc_fc(Rc4, rjk);
            F1 = orc_fc(Rc4, rij) * orc_dfc(Rc4, rik) * orc_fc(Rc4, rjk);
            F2 = orc_fc(Rc4, rij) * orc_fc(Rc4, rik) * orc_dfc(Rc4, rjk);
            for (n = 0; n < P->gt[3]; n++) ex[n] = exp(-P->gp[3][n] * (rij * rij + rik * rik + rjk * rjk));
            a52 = (1.0 / rik - c / rij) / rij;
            a62 = (1.0 / rij - c / rik) / rik;
            a53 = orc_fc(Rc4, rik) * orc_dfc(Rc4, rij) / rij;
            a63 = orc_fc(Rc4, rij) * orc_dfc(Rc4, rik) / rik;
            for (n = 0, g4 = 0; n < P->nsym; n++)
                if (P->gf[n][0] == 4) {
                    double zz = P->gp[5][P->gf[n][6]], lam = P->gp[6][P->gf[n][7]], eta = P->gp[3][P->gf[n][4]];
                    double base = 1.0 + lam * c;
                    double A2 = powz[P->gf[n][6]] * lam * zz * pow(base, zz - 1.0) * A0;
                    double A3 = powz[P->gf[n][6]] * pow(base, zz);
                    double B1 = ex[P->gf[n][4]], A1 = B1 * T0, A4 = -2.0 * eta * A0;
                    double B2 = A3 * A4 * T0, B3 = A2 * T0;
                    double A5 = A1 * (A2 * a52 + A3 * (a53 + A4)), A6 = A1 * (A2 * a62 + A3 * (a63 + A4));
                    int m = g4 + ind4[ds];
                    if (Fs)
                        for (q = 0; q < 3; q++) Fs[(size_t)m * 3 + q] -= 2.0 * (A5 * dij[q] + A6 * dik[q]);
                    if (Sn) {
                        double cj = B2 - c * B3 / (rij * rij) + A3 * F0 / rij;
                        double ck = B2 - c * B3 / (rik * rik) + A3 * F1 / rik;
                        double cjk = B2 + A3 * F2 / rjk;
                        double cx = B3 / (rij * rik);
                        for (q = 0; q < 3; q++) {
                            double u = dij[q] - dik[q], uq = dq[q] - dqk[q];
                            Sn[(size_t)m * 6 + q] += 2.0 * B1 * (cj * dij[q] * dij[q] + ck * dik[q] * dik[q] + cjk * u * u +
                                                                 cx * 2.0 * dij[q] * dik[q]);
                            Sn[(size_t)m * 6 + q + 3] += 2.0 * B1 * (cj * dij[q] * dq[q] + ck * dik[q] * dqk[q] + cjk * u * uq +
                                                                     cx * (dij[q] * dqk[q] + dik[q] * dq[q]));
                        }
                    }
                    g4++;
                }
        }
    }
    *dnn_out = dnn;
    free(seen);
}

/* ------------------------------------------------------------------ */
/* MLP                                                                 */
/* ------------------------------------------------------------------ */

/* Forward pass for one atom (src/nmlp.c:367-399, 412-431) and the energy
 * gradient dE_i/dG_i (the inner sums of src/nmlp.c:437-479). */
static double orc_mlp(const orc_model *M, int s, const double *Gi, double *grad) {
    const int *nu = M->nu;
    double a0[1024], h1[64], h2[64], d1[64], d2[64], e;
    int n, m, l;
    for (n = 0; n < nu[0]; n++) a0[n] = Gi[n] - M->Rmin[s][n] * M->DR[s][n];
    for (m = 0; m < nu[1]; m++) {
        double b = M->B[s][0][m];
        for (n = 0; n < nu[0]; n++) b += a0[n] * M->W[s][0][m * nu[0] + n];
        h1[m] = tanh(b);
        d1[m] = 1.0 - h1[m] * h1[m];
    }
    for (m = 0; m < nu[2]; m++) {
        double b = M->B[s][1][m];
        for (n = 0; n < nu[1]; n++) b += h1[n] * M->W[s][1][m * nu[1] + n];
        h2[m] = tanh(b);
        d2[m] = 1.0 - h2[m] * h2[m];
    }
    e = M->B[s][2][0];
    for (n = 0; n < nu[2]; n++) e += h2[n] * M->W[s][2][n];
    if (grad) {
        for (l = 0; l < nu[0]; l++) grad[l] = 0.0;
        for (m = 0; m < nu[2]; m++) {
            double tm = M->W[s][2][m] * d2[m];
            for (n = 0; n < nu[1]; n++) {
                double tn = tm * M->W[s][1][m * nu[1] + n] * d1[n];
                for (l = 0; l < nu[0]; l++) grad[l] += tn * M->W[s][0][n * nu[0] + l];
            }
        }
    }
    return e;
}

/* ------------------------------------------------------------------ */
/* public entry points                                                 */
/* ------------------------------------------------------------------ */

static void orc_lat(const double *lat9, double L[3][3]) {
    int a, b;
    for (a = 0; a < 3; a++)
        for (b = 0; b < 3; b++) L[a][b] = lat9[3 * a + b];
}

/* Neighbour list in the reference's layout.  X is wrapped in place when ND>0.
 * Returns 0, or -1 on neighbour overflow. */
int orc_nlist(const orc_model *M, int N, int NM, int ND, const double *lat9, double *X, double rc, int *nn,
              int *nj, int *nic, double *nr) {
    double L[3][3];
    orc_list T;
    int i, c, rv;
    orc_lat(lat9, L);
    if (ND > 0) orc_wrap(N, X, L);
    rv = orc_build_list(N, NM, ND, X, L, rc > 0 ? rc : M->rc_list, &T);
    if (rv == 0)
        for (i = 0; i < N; i++) {
            nn[i] = T.nn[i];
            for (c = 0; c < T.nn[i]; c++) {
                size_t o = (size_t)i * NM + c;
                nj[o] = T.j[o];
                nic[3 * o] = T.ic[3 * o]; nic[3 * o + 1] = T.ic[3 * o + 1]; nic[3 * o + 2] = T.ic[3 * o + 2];
                nr[o] = T.r[o];
            }
        }
    orc_list_free(&T);
    return rv;
}

/* Descriptors G[N*D] for one structure. */
int orc_descriptors_api(const orc_model *M, int N, int NM, int ND, const int *atmn, const double *lat9, double *X,
                        double *G) {
    double L[3][3];
    orc_list T;
    orc_lat(lat9, L);
    if (ND > 0) orc_wrap(N, X, L);
    if (orc_build_list(N, NM, ND, X, L, M->rc_list, &T)) { orc_list_free(&T); return -1; }
    orc_descriptors(M, &T, atmn, G);
    orc_list_free(&T);
    return 0;
}

/* Derivative blocks of one atom in the parse-file layout (src/nprs.c:419-431). */
int orc_fn_api(const orc_model *M, int N, int NM, int ND, const int *atmn, const double *lat9, double *X, int atom,
               int *dnn, int *dni, double *Fn, double *Sn) {
    double L[3][3];
    orc_list T;
    orc_lat(lat9, L);
    if (ND > 0) orc_wrap(N, X, L);
    if (orc_build_list(N, NM, ND, X, L, M->rc_list, &T)) { orc_list_free(&T); return -1; }
    orc_derivatives(M, &T, atmn, atom, dnn, dni, Fn, Sn);
    orc_list_free(&T);
    return 0;
}

/* Vector-Jacobian product of the descriptor map: for per-atom weights g[N*D],
 *   F[i] = -sum_j sum_m g[j][m] dG_j,m/dx_i,  U = -sum_i sum_m g[i][m] Sn_i,m
 * built from the materialised reference blocks (src/nmlp.c:433-479). */
int orc_vjp_api(const orc_model *M, int N, int NM, int ND, const int *atmn, const double *lat9, double *X,
                const double *g, double *F, double *U) {
    double L[3][3], *Fn, *Sn;
    int *dni, i, q, D = M->D;
    orc_list T;
    orc_lat(lat9, L);
    if (ND > 0) orc_wrap(N, X, L);
    if (orc_build_list(N, NM, ND, X, L, M->rc_list, &T)) { orc_list_free(&T); return -1; }
    Fn = (double *)malloc(sizeof(double) * (size_t)(NM + 1) * D * 3);
    Sn = (double *)malloc(sizeof(double) * (size_t)D * 6);
    dni = (int *)malloc(sizeof(int) * (NM + 1));
    for (q = 0; q < 6; q++) U[q] = 0.0;
    for (i = 0; i < N; i++) {
        int dnn, slot, m;
        orc_derivatives(M, &T, atmn, i, &dnn, dni, Fn, Sn);
        for (q = 0; q < 3; q++) F[3 * i + q] = 0.0;
        for (slot = 0; slot <= dnn; slot++) {
            int owner = slot < dnn ? dni[slot] : i;
            for (m = 0; m < D; m++)
                for (q = 0; q < 3; q++) F[3 * i + q] -= Fn[((size_t)slot * D + m) * 3 + q] * g[(size_t)owner * D + m];
        }
        for (m = 0; m < D; m++)
            for (q = 0; q < 6; q++) U[q] -= Sn[(size_t)m * 6 + q] * g[(size_t)i * D + m];
    }
    free(Fn); free(Sn); free(dni);
    orc_list_free(&T);
    return 0;
}

/* Energy (and optionally forces and virial) of one structure, following
 * CELL_ENE / CELL_FRC (src/cmod.c:128-191).  urep > 0 adds the short-range
 * repulsion (src/cmod.c:61-126).  p_gpa is the external pressure in GPa.
 * Returns 0, or -1 on neighbour overflow.  X is wrapped in place (ND>0). */
int orc_efs_api(const orc_model *M, int N, int NM, int ND, const int *atmn, const double *lat9, double *X,
                double urep, double p_gpa, int want_forces, double *E_out, double *H_out, double *EA, double *F,
                double *U) {
    double L[3][3], *G, *grad = NULL, E = 0.0;
    int i, q, D = M->D;
    orc_list T;
    orc_lat(lat9, L);
    if (ND > 0) orc_wrap(N, X, L);
    if (orc_build_list(N, NM, ND, X, L, M->rc_list, &T)) { orc_list_free(&T); return -1; }
    G = (double *)malloc(sizeof(double) * (size_t)N * D);
    orc_descriptors(M, &T, atmn, G);
    if (want_forces) grad = (double *)malloc(sizeof(double) * (size_t)N * D);
    for (i = 0; i < N; i++) {
        double e = orc_mlp(M, atmn[i], G + (size_t)i * D, grad ? grad + (size_t)i * D : NULL);
        if (EA) EA[i] = e;
        E += e;
    }
    if (want_forces) {
        double *Fn = (double *)malloc(sizeof(double) * (size_t)(T.NM + 1) * D * 3);
        double *Sn = (double *)malloc(sizeof(double) * (size_t)D * 6);
        int *dni = (int *)malloc(sizeof(int) * (T.NM + 1));
        for (q = 0; q < 6; q++) U[q] = 0.0;
        for (i = 0; i < N; i++) {
            int dnn, slot, m;
            orc_derivatives(M, &T, atmn, i, &dnn, dni, Fn, Sn);
            for (q = 0; q < 3; q++) F[3 * i + q] = 0.0;
            for (slot = 0; slot <= dnn; slot++) {
                int owner = slot < dnn ? dni[slot] : i;
                for (m = 0; m < D; m++)
                    for (q = 0; q < 3; q++)
                        F[3 * i + q] -= Fn[((size_t)slot * D + m) * 3 + q] * grad[(size_t)owner * D + m];
            }
            for (m = 0; m < D; m++)
                for (q = 0; q < 6; q++) U[q] -= Sn[(size_t)m * 6 + q] * grad[(size_t)i * D + m];
        }
        free(Fn); free(Sn); free(dni);
    }
    if (urep > 0.0) {
        /* CELL_UREP: ordered pairs closer than the sum of the species' minimum distances */
        for (i = 0; i < N; i++) {
            int c;
            for (c = 0; c < T.nn[i]; c++) {
                size_t o = (size_t)i * T.NM + c;
                double R = orc_mindist[M->spcz[atmn[i]]] + orc_mindist[M->spcz[atmn[T.j[o]]]], r = T.r[o];
                if (r < R) {
                    double fcv = r > R ? 0.0 : 0.5 * (1.0 + cos(ORC_PI * r / R));
                    double dfcv = r > R ? 0.0 : -0.5 * sin(ORC_PI * r / R) * ORC_PI / R;
                    E += urep * fcv * R / r;
                    if (want_forces) {
                        double t = -2.0 * urep * R / (r * r) * (-fcv / r + dfcv);
                        const double *d = T.d + 3 * o;
                        for (q = 0; q < 3; q++) F[3 * i + q] -= t * d[q];
                        for (q = 0; q < 3; q++) U[q] += 0.5 * t * d[q] * d[q];
                        for (q = 0; q < 3; q++) U[q + 3] += 0.5 * t * d[q] * d[(q + 1) % 3];
                    }
                }
            }
        }
    }
    if (want_forces) {
        for (i = 0; i < 3 * N; i++)
            if (fabs(F[i]) < 1e-8) F[i] = 0.0;
        for (q = 0; q < 6; q++)
            if (fabs(U[q]) < 1e-8) U[q] = 0.0;
    }
    *E_out = E;
    *H_out = E;
    if (ND == 3) *H_out += p_gpa / ORC_EV2GPA * orc_cell_volume(L);
    free(G);
    free(grad);
    orc_list_free(&T);
    return 0;
}
