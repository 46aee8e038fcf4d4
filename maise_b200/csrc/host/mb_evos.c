/*
 * mb_evos.c -- the evolutionary search's hand-off around the population
 * relax: the files one relaxed member leaves in EVOS/Gnnn/Mppp (RELX_INT,
 * src/emod.c:521-548, each member through CELL_RELX) and the ranking of a
 * generation (RANK_TR, src/emod.c:304-393).
 *
 * Per member directory:
 *   POSCAR.0   the structure before relaxation  \  SAVE_CELL's layout
 *   CONTCAR.0  the relaxed structure            /  (src/util.c:991-1060)
 *   OSZICAR.0  one enthalpy line per output; RELX_TR reads the last one
 *              (Read_OSZI, src/util.c:1130-1147: the number after column 27)
 *   OUTCAR.0   the final-state block of CELL_OUT (src/cmod.c:617-685)
 * RELX_TR (src/emod.c:710-718) reads CONTCAR.0 with READ_CELL and OSZICAR.0
 * with Read_OSZI, so a generation relaxed here continues in the
 * reference's EA loop unchanged.
 */
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <sys/types.h>

#include "../../../include/maise_b200.h"

#define MB_EV2GPA 160.2176565 /* src/util.c:8 */

int mb_handle_fail(int code, const char *msg);

/* chemical symbols by atomic number (1..100) */
static const char *const kSymbols[] = {
    "--", "H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg", "Al", "Si", "P",  "S",
    "Cl", "Ar", "K",  "Ca", "Sc", "Ti", "V",  "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As",
    "Se", "Br", "Kr", "Rb", "Sr", "Y",  "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn",
    "Sb", "Te", "I",  "Xe", "Cs", "Ba", "La", "Ce", "Pr", "Nd", "Pm", "Sm", "Eu", "Gd", "Tb", "Dy", "Ho",
    "Er", "Tm", "Yb", "Lu", "Hf", "Ta", "W",  "Re", "Os", "Ir", "Pt", "Au", "Hg", "Tl", "Pb", "Bi", "Po",
    "At", "Rn", "Fr", "Ra", "Ac", "Th", "Pa", "U",  "Np", "Pu", "Am", "Cm", "Bk", "Cf", "Es", "Fm"};

static const char *symbol(int z) { return (z >= 1 && z <= 100) ? kSymbols[z] : "--"; }

static int mkdir_p(const char *path) {
    char buf[1024];
    size_t n = strlen(path);
    if (n >= sizeof(buf)) return -1;
    memcpy(buf, path, n + 1);
    for (size_t k = 1; k <= n; k++)
        if (buf[k] == '/' || buf[k] == '\0') {
            const char c = buf[k];
            buf[k] = '\0';
            if (mkdir(buf, 0755) != 0 && errno != EEXIST) return -1;
            buf[k] = c;
        }
    return 0;
}

static void reciprocal_rows(const double *L, double *R) {
    double t;
    int k;
    R[6] = L[1] * L[5] - L[2] * L[4];
    R[7] = L[2] * L[3] - L[0] * L[5];
    R[8] = L[0] * L[4] - L[1] * L[3];
    R[0] = L[4] * L[8] - L[5] * L[7];
    R[1] = L[5] * L[6] - L[3] * L[8];
    R[2] = L[3] * L[7] - L[4] * L[6];
    R[3] = L[7] * L[2] - L[8] * L[1];
    R[4] = L[8] * L[0] - L[6] * L[2];
    R[5] = L[6] * L[1] - L[7] * L[0];
    t = 1.0 / (L[0] * L[4] * L[8] + L[1] * L[5] * L[6] + L[2] * L[3] * L[7] - L[0] * L[5] * L[7] -
               L[1] * L[3] * L[8] - L[2] * L[4] * L[6]);
    for (k = 0; k < 9; k++) R[k] *= t;
}

static double volume(const double *L) {
    return fabs(L[0] * L[4] * L[8] + L[2] * L[3] * L[7] + L[1] * L[5] * L[6] - L[0] * L[5] * L[7] -
                L[1] * L[3] * L[8] - L[2] * L[4] * L[6]);
}

/* A POSCAR in SAVE_CELL's layout: tag, scale 1, lattice rows, species
 * symbols and counts, "direct" and fractional coordinates, 14 decimals. */
static int write_poscar(const char *path, const char *tag, int N, int nspc, const int *spcz, const int *atmn,
                        const double *lat, const double *x) {
    FILE *f = fopen(path, "w");
    double R[9];
    int cnt[8] = {0}, i, q, s;
    if (!f) return -1;
    for (i = 0; i < N; i++) cnt[atmn[i]]++;
    fprintf(f, "%s\n", tag);
    fprintf(f, "% 17.14lf\n", 1.0);
    for (i = 0; i < 3; i++) {
        for (q = 0; q < 3; q++) fprintf(f, "% 19.14lf ", lat[3 * i + q]);
        fprintf(f, "\n");
    }
    for (s = 0; s < nspc; s++)
        if (cnt[s] > 0) fprintf(f, "%s ", symbol(spcz[s]));
    fprintf(f, "\n");
    for (s = 0; s < nspc; s++)
        if (cnt[s] > 0) fprintf(f, "%d ", cnt[s]);
    fprintf(f, "\ndirect\n");
    reciprocal_rows(lat, R);
    for (i = 0; i < N; i++) {
        for (q = 0; q < 3; q++) {
            const double fr = x[3 * i] * R[3 * q] + x[3 * i + 1] * R[3 * q + 1] + x[3 * i + 2] * R[3 * q + 2];
            fprintf(f, "% 19.14lf ", fr);
        }
        fprintf(f, "\n");
    }
    return fclose(f) ? -1 : 0;
}

int mb_evos_write(const char *evos_dir, int gen, int member, int N, int nspc, const int *spcz, const int *atmn,
                  const double *lat0, const double *x0, const double *lat, const double *x, double H, double E,
                  double p_gpa, const double *frc, const double *str, int iters) {
    char dir[1024], path[1100];
    FILE *f;
    int i, s;
    if (!evos_dir || N < 1 || nspc < 1 || nspc > 8 || !spcz || !atmn || !lat0 || !x0 || !lat || !x || gen < 0 ||
        member < 0)
        return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    for (i = 0; i < N; i++) {
        if (atmn[i] < 0 || atmn[i] >= nspc) return mb_handle_fail(MB_ERR_ARG, "species index out of range");
        if (i > 0 && atmn[i] < atmn[i - 1])
            return mb_handle_fail(MB_ERR_ARG, "atoms must be grouped by species (SAVE_CELL, src/util.c:1001-1006)");
    }
    if (snprintf(dir, sizeof(dir), "%s/G%03d/M%03d", evos_dir, gen, member) >= (int)sizeof(dir) || mkdir_p(dir))
        return mb_handle_fail(MB_ERR_ARG, "cannot create the member directory");
    snprintf(path, sizeof(path), "%s/POSCAR.0", dir);
    if (write_poscar(path, "B200", N, nspc, spcz, atmn, lat0, x0)) return mb_handle_fail(MB_ERR_ARG, "cannot write POSCAR.0");
    snprintf(path, sizeof(path), "%s/CONTCAR.0", dir);
    if (write_poscar(path, "B200", N, nspc, spcz, atmn, lat, x)) return mb_handle_fail(MB_ERR_ARG, "cannot write CONTCAR.0");
    /* OSZICAR: the enthalpy line CELL_OUT appends (src/cmod.c:682-685) */
    snprintf(path, sizeof(path), "%s/OSZICAR.0", dir);
    if (!(f = fopen(path, "w"))) return mb_handle_fail(MB_ERR_ARG, "cannot write OSZICAR.0");
    fprintf(f, "                            % 1.8lf\n", H);
    if (fclose(f)) return mb_handle_fail(MB_ERR_ARG, "cannot write OSZICAR.0");
    /* OUTCAR: the final-state block of CELL_OUT */
    snprintf(path, sizeof(path), "%s/OUTCAR.0", dir);
    if (!(f = fopen(path, "w"))) return mb_handle_fail(MB_ERR_ARG, "cannot write OUTCAR.0");
    {
        const char *b = "----------------------------------------------------------------------------------------------"
                        "------------\n";
        const double V = volume(lat);
        int cnt[8] = {0};
        for (i = 0; i < N; i++) cnt[atmn[i]]++;
        fprintf(f, "%s    Cell optimization    with libmaise_b200 (batched relax)\n%s", b, b);
        fprintf(f, "   relaxation type         3\n");
        fprintf(f, "   target pressure         %1.2lf GPa\n", p_gpa);
        fprintf(f, "   dimensionality          3\n");
        fprintf(f, "   species                ");
        for (s = 0; s < nspc; s++) fprintf(f, " %s    ", symbol(spcz[s]));
        fprintf(f, "\n   atoms of each species  ");
        for (s = 0; s < nspc; s++) fprintf(f, " %d    ", cnt[s]);
        fprintf(f, "\n   total number of atoms   %d\n%s\n\n\n", N, b);
        fprintf(f, "%s                   LATTICE VECTORS                                                 VOLUME (Angst^3/atom) \n%s",
                b, b);
        fprintf(f, "      % 12.6lf  % 12.6lf  % 12.6lf  % 45.6lf vol\n", lat[0], lat[1], lat[2], V / (double)N);
        fprintf(f, "      % 12.6lf  % 12.6lf  % 12.6lf\n", lat[3], lat[4], lat[5]);
        fprintf(f, "      % 12.6lf  % 12.6lf  % 12.6lf\n", lat[6], lat[7], lat[8]);
        if (frc) {
            fprintf(f, "%s                 POSITION (Angst)                     TOTAL-FORCE (eV/Angst)\n%s", b, b);
            for (i = 0; i < N; i++)
                fprintf(f, "   % 12.6lf % 12.6lf % 12.6lf   % 12.6lf % 12.6lf % 12.6lf\n", x[3 * i], x[3 * i + 1],
                        x[3 * i + 2], frc[3 * i], frc[3 * i + 1], frc[3 * i + 2]);
            fprintf(f, "%s", b);
        }
        if (str) {
            fprintf(f, "  Total   ");
            for (i = 0; i < 6; i++) fprintf(f, "% 15.8lf ", str[i] / V);
            fprintf(f, "\n  in kB   ");
            for (i = 0; i < 6; i++) fprintf(f, "% 15.8lf ", str[i] * MB_EV2GPA * 10.0 / V);
            fprintf(f, "\n%s", b);
        }
        fprintf(f, "  iter %3d   total enthalpy= % 14.8lf   energy=  % 14.8lf   % 14.8lf  % 14.8lf\n%s\n\n\n", iters, H,
                E, H / (double)N, E / (double)N, b);
    }
    if (fclose(f)) return mb_handle_fail(MB_ERR_ARG, "cannot write OUTCAR.0");
    return MB_OK;
}

typedef struct {
    double e;
    int p;
} rank_item;

static int cmp_rank(const void *a, const void *b) {
    const rank_item *x = (const rank_item *)a, *y = (const rank_item *)b;
    if (x->e < y->e) return -1;
    if (x->e > y->e) return 1;
    return x->p - y->p; /* equal enthalpies keep the member order */
}

int mb_evos_rank(int M, const double *H, const int *nat, int per_atom, int *order, double *fit) {
    rank_item *it;
    double emin = INFINITY, emax = -INFINITY;
    int p;
    if (M < 1 || !H || !order || (per_atom && !nat)) return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    it = (rank_item *)malloc(sizeof(rank_item) * M);
    if (!it) return mb_handle_fail(MB_ERR_ARG, "out of memory");
    for (p = 0; p < M; p++) {
        it[p].e = per_atom ? H[p] / (double)nat[p] : H[p];
        it[p].p = p;
        if (it[p].e < emin) emin = it[p].e;
        if (it[p].e > emax) emax = it[p].e;
    }
    if (!(emax - emin >= 1e-12)) {
        free(it);
        return mb_handle_fail(MB_ERR_STATE, "the energy diversity is too small (src/emod.c:324-331)");
    }
    if (fit)
        for (p = 0; p < M; p++) fit[p] = 0.5 * (1.0 - tanh(2.0 * (it[p].e - emin) / (emax - emin) - 1.0));
    qsort(it, M, sizeof(rank_item), cmp_rank);
    for (p = 0; p < M; p++) order[p] = it[p].p;
    free(it);
    return MB_OK;
}

int mb_evos_duplicates(int M, const double *cxc, const double *H, const double *vol, double cut, double *fit) {
    int p, k;
    if (M < 1 || !cxc || !H || !vol || !fit) return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    /* COMP_CL (src/eutl.c:394-413) against every better-ranked member,
     * worst first; the first one above the cutoff marks a duplicate
     * (src/emod.c:358-367) */
    for (p = M - 1; p >= 1; p--)
        for (k = p - 1; k >= 0; k--) {
            const double dv = 0.5 * (vol[p] - vol[k]) / (vol[p] + vol[k]), de = H[p] - H[k];
            const double t = 0.8 * cxc[(size_t)p * M + k] + 0.1 * exp(-0.5 * de * de / (0.05 * 0.05)) +
                             0.1 * exp(-0.5 * dv * dv / (0.01 * 0.01));
            if (t > cut) {
                fit[p] *= 0.001 + (1.0 - t) * (1.0 - t);
                break;
            }
        }
    return MB_OK;
}
