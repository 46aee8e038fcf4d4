/*
 * mb_model.c -- reader for MAISE 'model' files.
 *
 * A model file holds a fixed-width header table, the input component range
 * table, the network weights and, appended, the descriptor 'basis'.  The
 * fields read and their meaning follow:
 *   READ_MODEL   src/util.c:1233-1335   species, layer sizes, NSYM
 *   READ_ANN     src/nutl.c:502-633     ranges, weights, input-scaling fold
 *   V2W          src/nmlp.c:591-608     weight order (biases first)
 *   Build_PRS    src/nprs.c:75-257      basis table, B2A scaling, pair mixing
 *   check_ver    src/util.c:1948-1996   format version >= 2.4
 * The result is packed into the device parameter block (mb_params) and one
 * contiguous weight buffer.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../mb_internal.h"

/* atomic masses (amu) by atomic number and minimum interatomic distances
 * (Angstrom) used by the short-range repulsion; physical data tables that
 * must agree with the reference (src/util.c:11,13). */
/* the smallest double t with sqrt(t) >= R (R > 0): s < t exactly when
 * sqrt(s) < R, since sqrt is correctly rounded and non-decreasing */
static double sqrt_threshold(double R) {
    double t = R * R;
    if (!(R > 0.0)) return 0.0;
    while (sqrt(t) < R) t = nextafter(t, INFINITY);
    while (t > 0.0 && sqrt(nextafter(t, 0.0)) >= R) t = nextafter(t, 0.0);
    return t;
}

static const double mb_atom_mass[96] = {
    0.0, 1.008, 4.002602, 6.94, 9.0121831, 10.81, 12.011, 14.007, 15.999, 18.99840316, 20.1797, 22.98976928,
    24.305, 26.9815384, 28.085, 30.973762, 32.06, 35.45, 39.948, 39.0983, 40.078, 44.955908, 47.867, 50.9415,
    51.9961, 54.938043, 55.845, 58.933194, 58.6934, 63.546, 65.38, 69.723, 72.63, 74.921595, 78.971, 79.904,
    83.798, 85.4678, 87.62, 88.90584, 91.224, 92.90637, 95.95, 98, 101.07, 102.90549, 106.42, 107.8682,
    112.414, 114.818, 118.71, 121.76, 127.6, 126.90447, 131.293, 132.9054519, 137.327, 138.90547, 140.116,
    140.90766, 144.242, 145, 150.36, 151.964, 157.25, 158.925354, 162.5, 164.930328, 167.259, 168.934218,
    173.045, 174.9668, 178.49, 180.94788, 183.84, 186.207, 190.23, 192.217, 195.084, 196.96657, 200.592,
    204.38, 207.2, 208.9804, 209, 210, 222, 223, 226, 227, 232.0377, 231.03588, 238.02891, 237, 244, 243};
static const double mb_min_dist[96] = {
    0.0, 1.0, 1.0, 1.040, 0.773, 0.584, 0.499, 1.0, 1.0, 1.0, 1.0, 1.266, 1.114, 1.0, 1.0, 1.0,
    1.0, 1.0, 1.0, 1.610, 1.366, 1.123, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 0.895, 1.0, 1.0,
    1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 0.979, 1.030,
    1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0,
    1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 0.984, 1.0,
    1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0};

double mb_atomic_mass(int z) { return (z > 0 && z < 96) ? mb_atom_mass[z] : 0.0; }

static double mb_mass_of_z(int z) { return mb_atomic_mass(z) * 103.6427; }

/* ---- whole-file line access ---- */
typedef struct {
    char *buf;
    char **line;
    int n;
} mb_lines;

static int lines_read(const char *path, mb_lines *L) {
    FILE *f = fopen(path, "rb");
    long sz;
    int cap = 1024, i;
    char *p;
    memset(L, 0, sizeof(*L));
    if (!f) return -1;
    fseek(f, 0, SEEK_END);
    sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    L->buf = (char *)malloc(sz + 2);
    if (fread(L->buf, 1, sz, f) != (size_t)sz) { fclose(f); free(L->buf); return -1; }
    fclose(f);
    L->buf[sz] = '\0';
    L->line = (char **)malloc(sizeof(char *) * cap);
    p = L->buf;
    while (*p) {
        char *e = strchr(p, '\n');
        if (L->n == cap) { cap *= 2; L->line = (char **)realloc(L->line, sizeof(char *) * cap); }
        L->line[L->n++] = p;
        if (!e) break;
        *e = '\0';
        p = e + 1;
    }
    /* strip carriage returns */
    for (i = 0; i < L->n; i++) {
        size_t k = strlen(L->line[i]);
        if (k && L->line[i][k - 1] == '\r') L->line[i][k - 1] = '\0';
    }
    return 0;
}

static void lines_free(mb_lines *L) {
    free(L->buf);
    free(L->line);
    memset(L, 0, sizeof(*L));
}

static int find_prefix(const mb_lines *L, int from, const char *key) {
    size_t k = strlen(key);
    int i;
    for (i = from; i < L->n; i++)
        if (strncmp(L->line[i], key, k) == 0) return i;
    return -1;
}

/* integers after column 26 of a header row */
static int header_ints(const char *s, int *v, int n) {
    const char *p = s + 26;
    int i, used;
    if (strlen(s) < 26) return -1;
    for (i = 0; i < n; i++) {
        if (sscanf(p, "%d%n", &v[i], &used) != 1) return -1;
        p += used;
    }
    return 0;
}

/* "|  maise version | maise.X.Y.Z |" -> 1000X + 100Y + Z */
static int model_version(const mb_lines *L) {
    int i = find_prefix(L, 0, "|  maise version"), v[3] = {0, 0, 0}, k = 0;
    const char *p;
    char tok[128];
    if (i < 0) return -1;
    p = strchr(L->line[i] + 1, '|');
    if (!p || sscanf(p + 1, "%127s", tok) != 1 || strncmp(tok, "maise.", 6) != 0) return -1;
    p = tok + 6;
    while (k < 3 && *p) {
        v[k++] = atoi(p);
        while (*p && *p != '.') p++;
        if (*p) p++;
    }
    return v[0] * 1000 + v[1] * 100 + v[2];
}

typedef struct {
    int gf[512][8];
    int gt[7];
    double gp[7][10];
} raw_block;

static int parse_block(const mb_lines *L, int at, int nsym, raw_block *b, int *next, char *err, size_t el) {
    double a, r;
    int n, k;
    char name[32];
    if (at >= L->n || sscanf(L->line[at], "%lf %lf", &a, &r) != 2) {
        snprintf(err, el, "basis: bad scale line %d", at + 1);
        return -1;
    }
    at += 4; /* scale line, blank, column header, blank */
    for (n = 0; n < nsym; n++, at++) {
        int idx;
        if (at >= L->n || sscanf(L->line[at], "%d %d %d %d %d %d %d %d %d", &idx, &b->gf[n][0], &b->gf[n][1],
                                 &b->gf[n][2], &b->gf[n][3], &b->gf[n][4], &b->gf[n][5], &b->gf[n][6],
                                 &b->gf[n][7]) != 9) {
            snprintf(err, el, "basis: bad function line %d", at + 1);
            return -1;
        }
    }
    at++; /* blank */
    for (n = 0; n < 7; n++, at++) {
        double *g = b->gp[n];
        memset(g, 0, sizeof(double) * 10);
        if (at >= L->n || sscanf(L->line[at], "%31s %d %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf", name, &b->gt[n],
                                 &g[0], &g[1], &g[2], &g[3], &g[4], &g[5], &g[6], &g[7], &g[8], &g[9]) < 3) {
            snprintf(err, el, "basis: bad parameter line %d", at + 1);
            return -1;
        }
        if (b->gt[n] < 1 || b->gt[n] > 10) {
            snprintf(err, el, "basis: bad parameter count on line %d", at + 1);
            return -1;
        }
    }
    /* B2A: distances in units of a*r, exponents in 1/(a*r)^2 (src/nprs.c:183-189) */
    for (n = 0; n < 2; n++)
        for (k = 0; k < 10; k++) b->gp[n][k] *= a * r;
    for (n = 2; n < 4; n++)
        for (k = 0; k < 10; k++) b->gp[n][k] /= a * a * r * r;
    *next = at;
    return 0;
}

static int parse_basis(const mb_lines *L, mb_model *m, char *err, size_t el) {
    raw_block *blk = (raw_block *)calloc(MB_NPAIR, sizeof(raw_block));
    mb_params *P = &m->P;
    int b2a = find_prefix(L, 0, "  B2A"), i, n, s, t, nsym = -1, at;
    if (b2a < 0) { snprintf(err, el, "no basis (B2A) section"); free(blk); return -1; }
    /* NSYM: rows between the four header lines and " Rc  ", less one blank (src/util.c:1306-1318) */
    for (i = b2a + 5; i < L->n; i++) {
        if (strncmp(L->line[i], " Rc  ", 5) == 0) break;
        nsym++;
    }
    if (i >= L->n || nsym < 1 || nsym > 512) { snprintf(err, el, "basis: cannot count functions"); free(blk); return -1; }
    at = b2a + 1;
    for (s = 0; s < m->nspc; s++) {
        int next;
        if (parse_block(L, at, nsym, &blk[2 * s * s], &next, err, el)) { free(blk); return -1; }
        /* the following block starts two lines later; without one, the first block is reused
         * (src/nprs.c:222-231) */
        at = next + 2;
        if (at >= L->n) at = b2a + 1;
    }
    /* pair mixing for unlike species (src/nprs.c:233-252) */
    for (s = 0; s < m->nspc; s++)
        for (t = 0; t < m->nspc; t++)
            if (s != t) {
                raw_block *A = &blk[2 * s * s], *B = &blk[2 * t * t], *X = &blk[s * s + t * t];
                int k;
                memcpy(X->gf, blk[0].gf, sizeof(X->gf));
                memcpy(X->gt, blk[0].gt, sizeof(X->gt));
                for (n = 0; n < 2; n++)
                    for (k = 0; k < 10; k++) X->gp[n][k] = 0.5 * (A->gp[n][k] + B->gp[n][k]);
                for (n = 2; n < 4; n++)
                    for (k = 0; k < 10; k++)
                        X->gp[n][k] = pow(0.5 * (pow(A->gp[n][k], -0.5) + pow(B->gp[n][k], -0.5)), -2.0);
                for (n = 4; n < 7; n++)
                    for (k = 0; k < 10; k++) X->gp[n][k] = blk[0].gp[n][k];
            }
    /* function table of the species-0 block drives the layout */
    P->ng2 = P->ng4 = 0;
    for (n = 0; n < nsym; n++) {
        int type = blk[0].gf[n][0];
        if (type == 2) {
            if (P->ng4) { snprintf(err, el, "basis: G2 functions must precede G4 functions"); free(blk); return -1; }
            if (P->ng2 == MB_MAXG2) { snprintf(err, el, "basis: too many G2 functions"); free(blk); return -1; }
            P->ng2++;
        } else if (type == 4) {
            if (P->ng4 == MB_MAXG4) { snprintf(err, el, "basis: too many G4 functions"); free(blk); return -1; }
            P->ng4++;
        } else {
            snprintf(err, el, "basis: function type %d is not a G2/G4 Behler-Parrinello function", type);
            free(blk);
            return -1;
        }
    }
    {
        int c = m->nspc * (m->nspc + 1) / 2;
        if (P->ng2 * m->nspc + P->ng4 * c != m->nu[0]) {
            snprintf(err, el, "NCMP %d inconsistent with basis (%d)", m->nu[0], P->ng2 * m->nspc + P->ng4 * c);
            free(blk);
            return -1;
        }
    }
    P->nspc = m->nspc;
    P->D = m->nu[0];
    P->ne = blk[0].gt[3];
    P->nz = blk[0].gt[5];
    P->nlam = blk[0].gt[6];
    P->nzl = P->nz * P->nlam;
    if (P->nzl > MB_MAXZL) { snprintf(err, el, "basis: too many zeta/lambda combinations"); free(blk); return -1; }
    /* species-resolved block offsets (src/nprs.c:484-498) */
    {
        int a = P->ng2, b = P->ng4;
        memset(P->ind4, 0, sizeof(P->ind4));
        P->ind2[0] = 0; P->ind2[1] = a + b; P->ind2[2] = 2 * a + 3 * b; P->ind2[3] = 3 * a + 6 * b;
        P->ind4[0] = a; P->ind4[1] = 2 * a + b; P->ind4[2] = 2 * a + 2 * b; P->ind4[4] = 3 * a + 3 * b;
        P->ind4[8] = 3 * a + 4 * b; P->ind4[5] = 3 * a + 5 * b; P->ind4[9] = 4 * a + 6 * b;
        P->ind4[18] = 4 * a + 7 * b; P->ind4[10] = 4 * a + 8 * b; P->ind4[13] = 4 * a + 9 * b;
    }
    {
        const int (*gf)[8] = blk[0].gf;
        int g4first = P->ng2; /* index of the first G4 function */
        int p, f, e;
        for (s = 0; s < m->nspc; s++)
            for (t = 0; t < m->nspc; t++) {
                raw_block *W = &blk[s * s + t * t];
                p = s * s + t * t;
                P->f_rc2[p] = W->gp[0][gf[0][1]];
                P->f_rc4[p] = P->ng4 ? W->gp[0][gf[g4first][1]] : 0.0;
                P->f_rc4sq[p] = P->f_rc4[p] * P->f_rc4[p];
                P->f_rc4thr[p] = sqrt_threshold(P->f_rc4[p]);
                for (f = 0; f < P->ng2; f++) {
                    P->f_eta2[p][f] = W->gp[2][gf[f][3]];
                    P->f_rs[p][f] = W->gp[1][gf[f][2]];
                }
                for (e = 0; e < P->ne; e++) P->f_eta4[p][e] = W->gp[3][e];
            }
        P->d_rc2 = blk[0].gp[0][gf[0][1]];
        P->d_rc4 = P->ng4 ? blk[0].gp[0][gf[g4first][1]] : 0.0;
        P->d_rc4sq = P->d_rc4 * P->d_rc4;
        for (f = 0; f < P->ng2; f++) {
            P->d_eta2[f] = blk[0].gp[2][gf[f][3]];
            P->d_rs[f] = blk[0].gp[1][gf[f][2]];
        }
        for (e = 0; e < P->ne; e++) P->d_eta4[e] = blk[0].gp[3][e];
        P->zeta_int = 1;
        for (i = 0; i < P->nz; i++) {
            double z = blk[0].gp[5][i];
            P->zeta[i] = z;
            P->powz[i] = pow(2.0, 1.0 - z);
            if (!(z >= 1.0 && z <= 64.0 && z == floor(z))) P->zeta_int = 0;
            P->zbits[i] = (int)z;
            P->zm1bits[i] = (int)z - 1;
        }
        for (i = 0; i < P->nlam; i++) P->lam[i] = blk[0].gp[6][i];
        P->zeta_std = P->nz == 4 && P->zeta[0] == 1.0 && P->zeta[1] == 2.0 && P->zeta[2] == 4.0 && P->zeta[3] == 16.0;
        for (f = 0; f < P->ng4; f++) {
            const int *r = gf[g4first + f];
            if (r[4] >= P->ne || r[6] >= P->nz || r[7] >= P->nlam) {
                snprintf(err, el, "basis: G4 function %d indexes a missing parameter", g4first + f + 1);
                free(blk);
                return -1;
            }
            P->g4_e[f] = r[4];
            P->g4_zl[f] = r[6] * P->nlam + r[7];
        }
        /* neighbour-list cutoff: smallest Rc over all functions and species (src/nprs.c:455-462) */
        m->rc_list = blk[0].gp[0][0];
        for (s = 0; s < m->nspc; s++)
            for (n = 0; n < nsym; n++) {
                double rc = blk[2 * s * s].gp[0][gf[n][1]];
                if (m->rc_list > rc) m->rc_list = rc;
            }
    }
    free(blk);
    return 0;
}

void mb_model_free(mb_model *m) {
    free(m->weights);
    memset(m, 0, sizeof(*m));
}

int mb_model_load(const char *path, mb_model *m, char *err, size_t el) {
    mb_lines L;
    int i, s, k, n, r;
    double *V = NULL;
    memset(m, 0, sizeof(*m));
    if (lines_read(path, &L)) { snprintf(err, el, "cannot read model file '%s'", path); return -1; }
    if (L.n < 2 || !strstr(L.line[1], "neural")) { snprintf(err, el, "'%s' is not a neural-network model", path); goto fail; }
    if (model_version(&L) < 2400) { snprintf(err, el, "model format older than 2.4.00; convert the model first"); goto fail; }
    if ((i = find_prefix(&L, 0, "|  number of species    |")) < 0 || header_ints(L.line[i], &m->nspc, 1)) goto bad;
    if (m->nspc < 1 || m->nspc > MB_MAXSPC) { snprintf(err, el, "%d species; at most %d are supported", m->nspc, MB_MAXSPC); goto fail; }
    if ((i = find_prefix(&L, 0, "|  species types        |")) < 0 || header_ints(L.line[i], m->spcz, m->nspc)) goto bad;
    if ((i = find_prefix(&L, 0, "|  number of layers     |")) < 0 || header_ints(L.line[i], &m->nl, 1)) goto bad;
    if (m->nl != 4) { snprintf(err, el, "networks with exactly 2 hidden layers are supported (NL=%d)", m->nl); goto fail; }
    if ((i = find_prefix(&L, 0, "|  architecture         |")) < 0 || header_ints(L.line[i], m->nu, 4)) goto bad;
    if (m->nu[3] != 1 || m->nu[0] < 1 || m->nu[0] > MB_MAXD || m->nu[1] < 1 || m->nu[1] > MB_MAXH || m->nu[2] < 1 ||
        m->nu[2] > MB_MAXH) {
        snprintf(err, el, "unsupported architecture %d-%d-%d-%d", m->nu[0], m->nu[1], m->nu[2], m->nu[3]);
        goto fail;
    }
    if ((i = find_prefix(&L, 0, "|  number of weights    |")) < 0 || header_ints(L.line[i], &m->nw, 1)) goto bad;
    for (k = 0, n = 0; k < 3; k++) n += (m->nu[k] + 1) * m->nu[k + 1];
    if (m->nw != n * m->nspc) { snprintf(err, el, "weight count %d does not match the architecture", m->nw); goto fail; }
    if ((i = find_prefix(&L, 0, "        minimum          ")) < 0) goto bad;
    {
        int D = m->nu[0], h1 = m->nu[1], h2 = m->nu[2], net = MB_NET_SIZE(D, h1, h2);
        double *rmin = (double *)malloc(sizeof(double) * m->nspc * D), *dr = (double *)malloc(sizeof(double) * m->nspc * D);
        int row = i + 1, j;
        for (s = 0; s < m->nspc; s++)
            for (n = 0; n < D; n++, row++) {
                double mx;
                if (row >= L.n || sscanf(L.line[row], "%lf %lf %lf", &rmin[s * D + n], &mx, &dr[s * D + n]) != 3) {
                    free(rmin); free(dr);
                    goto bad;
                }
            }
        if ((i = find_prefix(&L, row, "|                        neural network weights")) < 0) { free(rmin); free(dr); goto bad; }
        V = (double *)malloc(sizeof(double) * m->nw);
        for (row = i + 2, j = 0; j < m->nw; row++) {
            if (row >= L.n || sscanf(L.line[row], "%lf", &V[j]) != 1) { free(rmin); free(dr); goto bad; }
            j++;
        }
        /* pack: per species [off | W0 | b0 | W1 | b1 | W2 | b2]; weight vector order is biases of all
         * layers, then weights [layer][out][in] (src/nmlp.c:591-608) */
        m->weights_len = (size_t)net * m->nspc;
        m->weights = (double *)calloc(m->weights_len, sizeof(double));
        for (s = 0, j = 0; s < m->nspc; s++) {
            double *w = m->weights + (size_t)s * net;
            double *off = w, *W0 = off + D, *b0 = W0 + h1 * D, *W1 = b0 + h1, *b1 = W1 + h2 * h1, *W2 = b1 + h2, *b2 = W2 + h2;
            m->P.w_off[s] = s * net;
            for (k = 0; k < h1; k++) b0[k] = V[j++];
            for (k = 0; k < h2; k++) b1[k] = V[j++];
            b2[0] = V[j++];
            for (k = 0; k < h1; k++)
                for (n = 0; n < D; n++) W0[k * D + n] = V[j++];
            for (k = 0; k < h2; k++)
                for (n = 0; n < h1; n++) W1[k * h1 + n] = V[j++];
            for (n = 0; n < h2; n++) W2[n] = V[j++];
            /* input-scaling fold (src/nutl.c:621-630) and the shift the MLP subtracts (src/nmlp.c:380) */
            for (k = 0; k < h1; k++)
                for (n = 0; n < D; n++) W0[k * D + n] *= dr[s * D + n];
            for (n = 0; n < D; n++) {
                double folded = rmin[s * D + n] / dr[s * D + n];
                off[n] = folded * dr[s * D + n];
            }
        }
        free(rmin);
        free(dr);
        m->P.h1 = h1;
        m->P.h2 = h2;
    }
    r = parse_basis(&L, m, err, el);
    if (r) goto fail;
    for (s = 0; s < m->nspc; s++) {
        int z = m->spcz[s];
        if (z < 1 || z > 95) { snprintf(err, el, "species %d has atomic number %d", s, z); goto fail; }
        m->P.rm[s] = mb_min_dist[z];
        m->mass[s] = mb_mass_of_z(z);
    }
    free(V);
    lines_free(&L);
    return 0;
bad:
    snprintf(err, el, "malformed model file '%s'", path);
fail:
    free(V);
    lines_free(&L);
    mb_model_free(m);
    return -1;
}
