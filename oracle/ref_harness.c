/*
 * ref_harness.c -- entry points into the reference MAISE sources compiled as
 * a CPU oracle (oracle/_ref/libmaise_ref.so).  TEST INFRASTRUCTURE ONLY: used
 * by tests/ to validate the C restatement (oracle/oracle.c) and the CUDA
 * path, and by bench.py as the reference CPU baseline.
 *
 * Every evaluation goes through the reference's own code: the first call of
 * a model runs CALL_MAISE (src/cmod.c:1164-1224), which reads ./model and
 * allocates the reference structures; later calls reuse them.  Relaxation
 * runs CELL_MIN (src/cmin.c:177-301) over the GSL stand-in of ref_shim.c.
 * The NVT loop restates the integrator of Dynamics (src/cmod.c:385-453)
 * around the reference CELL_FRC/CELL_KIN, because Dynamics itself writes
 * files every step and overflows its Lindemann arrays for N > NM
 * (src/cell.c:14-15, src/cmod.c:33-53).
 */
#include <omp.h>
#include <stddef.h>
#include <unistd.h>

#include "mlib.h"

extern long ECNTC, FCNTC; /* src/cmin.c:9 */

static ANN hR;
static PRS hP;
static PRS hW[9];
static LNK hL;
static Cell hC;
static int h_ready = 0, h_capN = 0, h_capNM = 0;
static char h_dir[1024];

/* CALL_MAISE in the model directory; (re)initialises when the model
 * directory changes or the structure outgrows the first call's arrays. */
static double h_call(const char *dir, int N, int NM, int ND, int NP, int XT, int *ATMN, double *LAT, double *X,
                     double *FRC, double *STR, double urep, double p_gpa) {
    char cwd[1024];
    double H;
    int reinit = !h_ready || N > h_capN || NM != h_capNM || strcmp(dir, h_dir) != 0;
    if (reinit) {
        /* arrays of a previous model are leaked on purpose: the reference never frees them */
        memset(&hR, 0, sizeof(hR));
        memset(&hP, 0, sizeof(hP));
        memset(hW, 0, sizeof(hW));
        memset(&hL, 0, sizeof(hL));
        memset(&hC, 0, sizeof(hC));
        hL.B = 0;
        if (!getcwd(cwd, sizeof(cwd))) return NAN;
        if (chdir(dir)) return NAN;
    }
    hR.UREP = urep;
    hC.p = p_gpa;
    H = CALL_MAISE(&hR, &hP, hW, &hL, &hC, 0, N, NM, ND, NP, XT, ATMN, LAT, X, FRC, STR);
    if (reinit) {
        if (chdir(cwd)) return NAN;
        h_ready = 1;
        h_capN = N;
        h_capNM = NM;
        snprintf(h_dir, sizeof(h_dir), "%s", dir);
    }
    return H;
}

/* the per-call field setup of CALL_MAISE (src/cmod.c:1170-1181) */
static void h_prologue(int N, int NM, int ND, int NP, double p_gpa, double urep) {
    hC.N = N;
    hC.NM = NM;
    hC.ND = ND;
    hC.NP = NP;
    hC.XT = 1;
    hC.R0 = 1.0;
    hR.JOBT = hC.JOBT = 20;
    hR.NB = hC.NB = 1;
    hR.A = hC.A = N;
    hR.NP = NP;
    hC.p = p_gpa / eV2GPa;
    hR.UREP = urep;
}

int ref_sizes(int *out) {
    out[0] = (int)sizeof(ANN);
    out[1] = (int)sizeof(PRS);
    out[2] = (int)sizeof(LNK);
    out[3] = (int)sizeof(Cell);
    out[4] = (int)offsetof(ANN, UREP);
    out[5] = (int)offsetof(LNK, B);
    out[6] = (int)offsetof(Cell, p);
    out[7] = (int)offsetof(Cell, E);
    out[8] = (int)offsetof(Cell, H);
    out[9] = (int)offsetof(Cell, N);
    return 10;
}

/* Energy, forces (FRC[3N]) and virial (STR[6]) through CALL_MAISE.
 * EA (per-atom energies) and E_out (energy without pV) may be NULL. */
double ref_efs(const char *dir, int N, int NM, int ND, int NP, int XT, int *ATMN, double *LAT, double *X, double urep,
               double p_gpa, double *FRC, double *STR, double *EA, double *E_out) {
    double H = h_call(dir, N, NM, ND, NP, XT, ATMN, LAT, X, FRC, STR, urep, p_gpa);
    int i;
    if (EA)
        for (i = 0; i < N; i++) EA[i] = hC.EA[i];
    if (E_out) *E_out = hC.E;
    return H;
}

/* Energy only (CELL_ENE, src/cmod.c:128-151) on Cartesian X. */
double ref_energy(const char *dir, int N, int NM, int ND, int NP, int *ATMN, double *LAT, double *X, double urep,
                  double p_gpa) {
    double *F = (double *)malloc(sizeof(double) * 3 * N), S[6];
    double *Xc = (double *)malloc(sizeof(double) * 3 * N), H;
    memcpy(Xc, X, sizeof(double) * 3 * N);
    if (!h_ready || strcmp(dir, h_dir) != 0 || N > h_capN || NM != h_capNM)
        h_call(dir, N, NM, ND, NP, 1, ATMN, LAT, Xc, F, S, urep, p_gpa);
    memcpy(Xc, X, sizeof(double) * 3 * N);
    h_prologue(N, NM, ND, NP, p_gpa, urep);
    CAST_CELL(&hC, ATMN, LAT, Xc);
    H = CELL_ENE(&hR, &hP, hW, &hC, &hL);
    free(F);
    free(Xc);
    return H;
}

/* Descriptors G[N*D] via PARS_STR/PRS_BP with all derivative blocks
 * computed (EFS = 3); ref_fn then reads one atom's blocks. */
int ref_descriptors(const char *dir, int N, int NM, int ND, int NP, int *ATMN, double *LAT, double *X, double *G) {
    double *F = (double *)malloc(sizeof(double) * 3 * N), S[6];
    double *Xc = (double *)malloc(sizeof(double) * 3 * N);
    int i, n;
    memcpy(Xc, X, sizeof(double) * 3 * N);
    if (!h_ready || strcmp(dir, h_dir) != 0 || N > h_capN || NM != h_capNM)
        h_call(dir, N, NM, ND, NP, 1, ATMN, LAT, Xc, F, S, 0.0, 0.0);
    memcpy(Xc, X, sizeof(double) * 3 * N);
    h_prologue(N, NM, ND, NP, 0.0, 0.0);
    CAST_CELL(&hC, ATMN, LAT, Xc);
    for (i = 0; i < N; i++) hL.MRK[i] = 1;
    hP.EFS = 3;
    PARS_STR(&hP, hW, &hC, &hL, 0, ".");
    for (i = 0; i < N; i++)
        for (n = 0; n < hP.D; n++) G[(size_t)i * hP.D + n] = hL.Cn[i][n];
    free(F);
    free(Xc);
    return hP.D;
}

/* The neighbour list of the reference's LIST (src/cell.c:82-185) for
 * Cartesian X: nn[N] counts, and per entry t of atom i the neighbour atom
 * nj[i*cap+t] and its integer image nic[(i*cap+t)*3+q].  LIST stores the
 * image as the Cartesian shift S = sum_q ic_q L_q (src/cell.c:127-131);
 * ic_q = rint(S . R_q) recovers the integers (R_q are the reciprocal rows
 * Reciprocal() set, L_p . R_q = delta_pq).  Xw[3N] receives the positions
 * after LIST's wrap.  Returns -1 if an atom has more than cap neighbours. */
int ref_nlist(const char *dir, int N, int NM, int ND, int NP, int *ATMN, double *LAT, double *X, int cap, int *nn,
              int *nj, int *nic, double *Xw) {
    double *F = (double *)malloc(sizeof(double) * 3 * N), S[6];
    double *Xc = (double *)malloc(sizeof(double) * 3 * N);
    int i, t, q, rv = 0;
    memcpy(Xc, X, sizeof(double) * 3 * N);
    if (!h_ready || strcmp(dir, h_dir) != 0 || N > h_capN || NM != h_capNM)
        h_call(dir, N, NM, ND, NP, 1, ATMN, LAT, Xc, F, S, 0.0, 0.0);
    memcpy(Xc, X, sizeof(double) * 3 * N);
    h_prologue(N, NM, ND, NP, 0.0, 0.0);
    CAST_CELL(&hC, ATMN, LAT, Xc);
    LIST(&hC, 0);
    for (i = 0; i < N && !rv; i++) {
        nn[i] = hC.Nn[i];
        if (nn[i] > cap) {
            rv = -1;
            break;
        }
        for (t = 0; t < nn[i]; t++) {
            size_t o = (size_t)i * cap + t;
            nj[o] = hC.Ni[i][t];
            for (q = 0; q < 3; q++) {
                double s = hC.S[i][t][0] * hC.R[q][0] + hC.S[i][t][1] * hC.R[q][1] + hC.S[i][t][2] * hC.R[q][2];
                nic[3 * o + q] = (int)lrint(s);
            }
        }
    }
    if (Xw)
        for (i = 0; i < N; i++)
            for (q = 0; q < 3; q++) Xw[3 * i + q] = hC.X[i][q];
    free(F);
    free(Xc);
    return rv;
}

/* Derivative blocks of one atom from the last ref_descriptors call, in the
 * parse-file layout: fn[(slot*D+m)*3+q], slot == dnn is the self block. */
int ref_fn(int atom, int *dnn, int *dni, double *fn, double *sn) {
    int j, m, q, D = hP.D;
    *dnn = hL.DNn[atom];
    for (j = 0; j <= *dnn; j++) {
        if (j < *dnn) dni[j] = hL.DNi[atom][j];
        for (m = 0; m < D; m++)
            for (q = 0; q < 3; q++) fn[((size_t)j * D + m) * 3 + q] = hL.Fn[atom][j][m][q];
    }
    if (sn)
        for (m = 0; m < D; m++)
            for (q = 0; q < 6; q++) sn[(size_t)m * 6 + q] = hL.Sn[atom][m][q];
    return 0;
}

/* Wrapped Cartesian positions after the last evaluation (LIST wraps, src/cell.c:90-91). */
int ref_positions(int N, double *X) {
    int i, q;
    for (i = 0; i < N; i++)
        for (q = 0; q < 3; q++) X[3 * i + q] = hC.X[i][q];
    return 0;
}

/* Cell relaxation through CELL_MIN (src/cmin.c:177-301).  On return X and
 * LAT hold the relaxed Cartesian positions and lattice; counts[0..2] =
 * energy calls, force calls, iterations. */
double ref_relax(const char *dir, int N, int NM, int ND, int NP, int *ATMN, double *LAT, double *X, double urep,
                 double p_gpa, int rlxt, int mitr, double etol, long *counts) {
    double *F = (double *)malloc(sizeof(double) * 3 * N), S[6];
    double *Xc = (double *)malloc(sizeof(double) * 3 * N), H;
    int i, q, nfree = 0;
    memcpy(Xc, X, sizeof(double) * 3 * N);
    if (!h_ready || strcmp(dir, h_dir) != 0 || N > h_capN || NM != h_capNM)
        h_call(dir, N, NM, ND, NP, 1, ATMN, LAT, Xc, F, S, urep, p_gpa);
    memcpy(Xc, X, sizeof(double) * 3 * N);
    h_prologue(N, NM, ND, NP, p_gpa, urep);
    CAST_CELL(&hC, ATMN, LAT, Xc);
    for (i = 0; i < N; i++)
        for (q = 0; q < 3; q++) hC.FF[i][q] = 1;
    hC.RLXT = rlxt;
    hR.MINT = 0;
    hC.MINT = 0;
    hR.MITR = mitr;
    hR.ETOL = etol;
    hR.FRAC = 0.0;
    hC.OUT = 0;
    hC.it = 0;
    JAR(&hC);
    CELL_FRC(&hR, &hP, hW, &hC, &hL);
    CELL_MIN(&hR, &hP, hW, &hC, &hL);
    H = hC.H;
    for (i = 0; i < N; i++)
        for (q = 0; q < 3; q++) X[3 * i + q] = hC.X[i][q];
    for (i = 0; i < 3; i++)
        for (q = 0; q < 3; q++) LAT[3 * i + q] = hC.L[i][q];
    counts[0] = ECNTC;
    counts[1] = FCNTC;
    counts[2] = hC.it;
    (void)nfree;
    free(F);
    free(Xc);
    return H;
}

/* NVT molecular dynamics: Maxwell initial velocities (src/cmod.c:224-280,
 * Park-Miller streams src/util.c:1829-1873 seeded by PlantSeeds(seed)),
 * then nsteps of the NVT branch of Dynamics (src/cmod.c:385-453):
 *   E+F+S, K, xi += dt/tau^2 (2K/(3 N T) - 1), x += v dt + f dt^2/2,
 *   v += f dt with f = F/m - xi v, wrap.
 * If V is non-NULL and vin != 0 the given velocities are used instead of
 * Maxwell's.  Hs[n], Ks[n] record H and K at the start of step n.  xi0 is
 * the thermostat variable at the start (0 for a new run).  On return X and
 * V hold the final state.  Returns the final xi. */
double ref_nvt(const char *dir, int N, int NM, int ND, int NP, int *ATMN, double *LAT, double *X, double *V, int vin,
               long seed, double T0, double dt, double tau, int nsteps, double urep, double *Hs, double *Ks,
               double xi0) {
    double *F = (double *)malloc(sizeof(double) * 3 * N), S[6];
    double *Xc = (double *)malloc(sizeof(double) * 3 * N);
    const double kbinv = 11604.0; /* src/cmod.c:5 */
    double T = T0 / kbinv, xi = xi0;
    int i, q, n;
    memcpy(Xc, X, sizeof(double) * 3 * N);
    if (!h_ready || strcmp(dir, h_dir) != 0 || N > h_capN || NM != h_capNM)
        h_call(dir, N, NM, ND, NP, 1, ATMN, LAT, Xc, F, S, urep, 0.0);
    memcpy(Xc, X, sizeof(double) * 3 * N);
    h_prologue(N, NM, ND, NP, 0.0, urep);
    CAST_CELL(&hC, ATMN, LAT, Xc);
    for (i = 0; i < N; i++)
        for (q = 0; q < 3; q++) hC.FF[i][q] = 1;
    if (vin && V) {
        for (i = 0; i < N; i++)
            for (q = 0; q < 3; q++) hC.V[i][q] = V[3 * i + q];
    } else {
        PlantSeeds(seed);
        Maxwell(&hC, T, 20);
    }
    if (ND > 0) JAR(&hC);
    for (n = 0; n < nsteps; n++) {
        double fs;
        hC.H = CELL_FRC(&hR, &hP, hW, &hC, &hL);
        hC.K = CELL_KIN(&hC);
        if (Hs) Hs[n] = hC.H;
        if (Ks) Ks[n] = hC.K;
        fs = 1.0 / (tau * tau) * (2.0 * hC.K / ((3.0 * (double)hC.N) * T) - 1.0);
        xi += dt * fs;
        for (i = 0; i < N; i++)
            for (q = 0; q < 3; q++) {
                double fi = hC.F[i][q] / hC.m[hC.ATMZ[i]] - xi * hC.V[i][q];
                hC.X[i][q] += hC.V[i][q] * dt + 0.5 * fi * dt * dt;
                hC.V[i][q] += fi * dt;
            }
        JAR(&hC);
    }
    for (i = 0; i < N; i++)
        for (q = 0; q < 3; q++) {
            X[3 * i + q] = hC.X[i][q];
            if (V) V[3 * i + q] = hC.V[i][q];
        }
    free(F);
    free(Xc);
    return xi;
}

/* Maxwell velocities only (for seeding the GPU integrator identically). */
int ref_maxwell(const char *dir, int N, int NM, int ND, int NP, int *ATMN, double *LAT, double *X, long seed, double T0,
                double *V) {
    double *F = (double *)malloc(sizeof(double) * 3 * N), S[6];
    double *Xc = (double *)malloc(sizeof(double) * 3 * N);
    int i, q;
    memcpy(Xc, X, sizeof(double) * 3 * N);
    if (!h_ready || strcmp(dir, h_dir) != 0 || N > h_capN || NM != h_capNM)
        h_call(dir, N, NM, ND, NP, 1, ATMN, LAT, Xc, F, S, 0.0, 0.0);
    memcpy(Xc, X, sizeof(double) * 3 * N);
    h_prologue(N, NM, ND, NP, 0.0, 0.0);
    CAST_CELL(&hC, ATMN, LAT, Xc);
    for (i = 0; i < N; i++)
        for (q = 0; q < 3; q++) hC.FF[i][q] = 1;
    PlantSeeds(seed);
    Maxwell(&hC, T0 / 11604.0, 20);
    for (i = 0; i < N; i++)
        for (q = 0; q < 3; q++) V[3 * i + q] = hC.V[i][q];
    free(F);
    free(Xc);
    return 0;
}

/* A POSCAR/CONTCAR read by the reference's READ_CELL (src/util.c:820-989)
 * into the harness cell (a model must be loaded, and the file's species must
 * be among its species): N, lattice rows, Cartesian positions and species
 * indices.  Returns 0, -1 if the file cannot be read, -2 if N > cap. */
int ref_read_cell(const char *path, int cap, int *N, double *lat, double *X, int *atmn) {
    int i, q;
    if (!h_ready) return -1;
    hC.A = h_capN;
    if (!READ_CELL(&hC, (char *)path)) return -1;
    *N = hC.N;
    if (hC.N > cap) return -2;
    for (i = 0; i < 3; i++)
        for (q = 0; q < 3; q++) lat[3 * i + q] = hC.L[i][q];
    for (i = 0; i < hC.N; i++) {
        atmn[i] = hC.ATMN[i];
        for (q = 0; q < 3; q++) X[3 * i + q] = hC.X[i][q];
    }
    return 0;
}

/* The enthalpy RELX_TR takes from an OSZICAR (Read_OSZI, src/util.c:1130-1147). */
double ref_read_oszi(const char *path) { return Read_OSZI((char *)path); }

/* RDF (src/cell.c:369-417) of one structure as RANK_TR computes it for
 * duplicate detection: LIST with the cutoff Rmax, then RDF(C, normalise),
 * with bins NRDF = 3000 over [0, rmax), Gaussian width sigma and taper from
 * rmin.  out[(pair * 3000 + k)] for the species pairs m <= n in row-major
 * order.  Returns the bin count. */
int ref_rdf(const char *dir, int N, int NM, int ND, int NP, int *ATMN, double *LAT, double *X, double rmin,
            double rmax, double sigma, int normalise, double *out) {
    double *F = (double *)malloc(sizeof(double) * 3 * N), S[6];
    double *Xc = (double *)malloc(sizeof(double) * 3 * N), rc;
    int k, m, n, pair;
    memcpy(Xc, X, sizeof(double) * 3 * N);
    if (!h_ready || strcmp(dir, h_dir) != 0 || N > h_capN || NM != h_capNM)
        h_call(dir, N, NM, ND, NP, 1, ATMN, LAT, Xc, F, S, 0.0, 0.0);
    memcpy(Xc, X, sizeof(double) * 3 * N);
    h_prologue(N, NM, ND, NP, 0.0, 0.0);
    CAST_CELL(&hC, ATMN, LAT, Xc);
    rc = hC.Rc;
    hC.Rc = rmax;
    hC.Rmax = rmax;
    hC.Rmin = rmin;
    hC.DR = sigma;
    LIST(&hC, 0);
    RDF(&hC, normalise);
    hC.Rc = rc;
    for (m = 0, pair = 0; m < hC.NSPC; m++)
        for (n = m; n < hC.NSPC; n++, pair++)
            for (k = 0; k < hC.NRDF; k++) out[(size_t)pair * hC.NRDF + k] = hC.RDF[k][m][n];
    free(F);
    free(Xc);
    return hC.NRDF;
}

/* A descriptor file read back by the reference's LNK_IN (src/nprs.c:308-377)
 * into a private LNK: hdr = {EFS, D, N, NF}, ehdr = {E, p, DE}, atmn[N],
 * Cn[N*D]; then ref_efile_block reads one marked atom's blocks and
 * ref_efile_sn the strain blocks. */
static LNK eL;
static int eEFS, eD, eScaled;
int ref_efile_read(const char *dir, int o, int *hdr, double *ehdr, int *atmn, double *Cn) {
    char buf[1200];
    FILE *in;
    int i, n, N, NF, DNn;
    snprintf(buf, sizeof(buf), "%s/e%06d", dir, o);
    if (!(in = fopen(buf, "r"))) return -1;
    if (fscanf(in, "%d %d %d %d %d", &eEFS, &eD, &N, &NF, &DNn) != 5) {
        fclose(in);
        return -1;
    }
    fclose(in);
    memset(&eL, 0, sizeof(eL));
    LNK_IN(&eL, o, (char *)dir);
    eScaled = 0;
    hdr[0] = eEFS;
    hdr[1] = eD;
    hdr[2] = eL.N;
    hdr[3] = eL.NF;
    ehdr[0] = eL.E;
    ehdr[1] = eL.p;
    ehdr[2] = eL.DE;
    for (i = 0; i < eL.N; i++) {
        atmn[i] = eL.ATMN[i];
        for (n = 0; n < eD; n++) Cn[(size_t)i * eD + n] = eL.Cn[i][n];
    }
    return 0;
}

/* Blocks of marked atom i from the last ref_efile_read: dnn, dni[dnn], the
 * reference force F[3] and fn[(slot*D+n)*3+q] with slot dnn the self block. */
int ref_efile_block(int i, int *dnn, int *dni, double *F, double *fn) {
    int j, n, q;
    if (!(eEFS == 1 || eEFS == 3) || !eL.MRK[i]) return -1;
    *dnn = eL.DNn[i];
    for (q = 0; q < 3; q++) F[q] = eL.F[i][q];
    for (j = 0; j <= *dnn; j++) {
        if (j < *dnn) dni[j] = eL.DNi[i][j];
        for (n = 0; n < eD; n++)
            for (q = 0; q < 3; q++) fn[((size_t)j * eD + n) * 3 + q] = eL.Fn[i][j][n][q];
    }
    return 0;
}

/* Strain blocks sn[(i*D+n)*6+k] and the reference stresses S[6]. */
int ref_efile_sn(double *sn, double *S) {
    int i, n, k;
    if (!(eEFS == 2 || eEFS == 3)) return -1;
    for (k = 0; k < 6; k++) S[k] = eL.S[k];
    for (i = 0; i < eL.N; i++)
        for (n = 0; n < eD; n++)
            for (k = 0; k < 6; k++) sn[((size_t)i * eD + n) * 6 + k] = eL.Sn[i][n][k];
    return 0;
}

/* The training terms of the last ref_efile_read structure through the
 * reference's own functions: the network V (V2W order, src/nmlp.c:591-608;
 * nspc species, D-h1-h2-1, tanh hidden layers) with input table rmin/dr
 * [nspc*D]; ADJT_LNK (src/nmod.c:244-259) puts Cn (and, for EFS 1, Fn) on
 * the input scale -- once per read; then
 *   E = FRC_ANN_PARA (src/nmlp.c:29-102), f[3N] the forces it leaves on
 *       the marked atoms (0 elsewhere),
 *   gE = DE_ANN_PARA's accumulation (src/nmlp.c:292-354) and
 *   gF = DF_ANN_PARA's (src/nmlp.c:104-290), each in dfunc_gsl's order
 *       (src/nmin.c:280-295: per species biases, then weights), not yet
 *       divided by the number of structures.
 * w is the structure's weight L->W. */
double ref_train_terms(int nspc, int D, int h1, int h2, const double *V, const double *rmin, const double *dr,
                       double WE, double WF, double w, double *f, double *gE, double *gF) {
    ANN R;
    int s, k, m, n, i, mx, dnm = 0;
    double E, ***e, ***d, ***c, ***xn, ***xm, ***Bp, ****Wp;
    if (eD != D) return NAN;
    memset(&R, 0, sizeof(R));
    R.NSPC = nspc;
    R.D = D;
    R.NL = 4;
    R.NU[0] = D; R.NU[1] = h1; R.NU[2] = h2; R.NU[3] = 1;
    R.GT[0] = 0; R.GT[1] = 1; R.GT[2] = 1; R.GT[3] = 0;
    R.MIX = 0;
    R.O = 0;
    R.STR = 1;
    R.EFS = eEFS;
    R.WE = WE;
    R.WF = WF;
    mx = D > h1 ? D : h1;
    if (h2 > mx) mx = h2;
    R.B = make_d3D(nspc, 3, mx);
    R.W = make_d4D(nspc, 3, mx, mx);
    R.Rmin = make_d2D(nspc, D);
    R.DR = make_d2D(nspc, D);
    for (s = 0; s < nspc; s++)
        for (n = 0; n < D; n++) {
            R.Rmin[s][n] = rmin[s * D + n];
            R.DR[s][n] = dr[s * D + n];
        }
    V2W(&R, (double *)V);
    if (!eScaled) {
        /* Build_LNK leaves DNs unset for unmarked atoms (src/nutl.c:379-387)
         * and ADJT_LNK indexes DR with DNs[i][0] of every atom
         * (src/nmod.c:254-257): give those unused rows a valid species */
        if (eEFS == 1 || eEFS == 3)
            for (i = 0; i < eL.N; i++)
                if (!eL.MRK[i]) eL.DNs[i][0] = eL.ATMN[i];
        ADJT_LNK(&R, &eL);
        eScaled = 1;
    }
    eL.W = w;
    for (i = 0; i < eL.N; i++)
        if (eL.DNn[i] > dnm) dnm = eL.DNn[i];
    e = make_d3D(eL.N, 4, mx);
    d = make_d3D(eL.N, 4, mx);
    c = make_d3D(eL.N, 4, mx);
    xn = make_d3D(mx, dnm + 1, 3);
    xm = make_d3D(mx, dnm + 1, 3);
    Bp = make_d3D(nspc, 3, mx);
    Wp = make_d4D(nspc, 3, mx, mx);
    E = FRC_ANN_PARA(&R, &eL, e, d);
    for (i = 0; i < eL.N; i++)
        for (k = 0; k < 3; k++) f[3 * i + k] = ((eEFS == 1 || eEFS == 3) && eL.MRK[i]) ? eL.f[i][k] : 0.0;
    for (int pass = 0; pass < 2; pass++) {
        double *out = pass ? gF : gE;
        int o = 0;
        for (s = 0; s < nspc; s++)
            for (k = 0; k < 3; k++)
                for (m = 0; m < mx; m++) {
                    Bp[s][k][m] = 0.0;
                    for (n = 0; n < mx; n++) Wp[s][k][m][n] = 0.0;
                }
        if (pass == 0)
            DE_ANN_PARA(&R, &eL, Bp, Wp, e);
        else if (eEFS == 1 || eEFS == 3)
            DF_ANN_PARA(&R, &eL, Bp, Wp, e, d, c, xn, xm);
        for (s = 0; s < nspc; s++) {
            for (k = 0; k < 3; k++)
                for (m = 0; m < R.NU[k + 1]; m++) out[o++] = Bp[s][k][m];
            for (k = 0; k < 3; k++)
                for (m = 0; m < R.NU[k + 1]; m++)
                    for (n = 0; n < R.NU[k]; n++) out[o++] = Wp[s][k][m][n];
        }
    }
    free_d3D(e, eL.N, 4);
    free_d3D(d, eL.N, 4);
    free_d3D(c, eL.N, 4);
    free_d3D(xn, mx, dnm + 1);
    free_d3D(xm, mx, dnm + 1);
    free_d3D(Bp, nspc, 3);
    free_d4D(Wp, nspc, 3, mx);
    free_d3D(R.B, nspc, 3);
    free_d4D(R.W, nspc, 3, mx);
    free_d2D(R.Rmin, nspc);
    free_d2D(R.DR, nspc);
    return E;
}
