/*
 * mb_parse.c -- the parse path: one structure's descriptor file e%06d in
 * the layout LNK_OUT writes (src/nprs.c:380-442) and LNK_IN reads
 * (src/nprs.c:308-377), the input of the reference's network training
 * (PARS_DAT, src/nprs.c:983-1366).
 *
 *   header   EFS D N NF DNn E p DE
 *   [EFS 1,3] the indices of the marked atoms (force training)
 *   [EFS 2,3] the structure's reference stresses
 *   the data path, then per atom its species and D descriptors
 *   [EFS 1,3] per marked atom i: i, DNn_i and its reference force, the
 *             block dG_i/dx_i, then for each neighbour atom j its index and
 *             the block dG_j/dx_i (D rows of 3)
 *   [EFS 2,3] per atom the D rows of dG/dstrain (xx yy zz xy yz zx)
 *
 * The descriptors come from mb_descriptors and every derivative block from
 * the descriptor tangent (mb_descriptor_jvp): a unit displacement of atom i
 * along axis q gives column q of all of i's blocks at once; a unit
 * deformation gives one strain column of every atom.  The neighbour atoms
 * of a marked atom are listed in ascending index (the reference lists them
 * in its neighbour-list order).  An atom that is its own periodic neighbour
 * has one self block holding the whole dG_i/dx_i; the reference keeps the
 * part that comes through i's images in a second block listed under i's
 * own index.  The contraction the force training makes of the blocks
 * (FRC_ANN, src/nmlp.c:433-479) is the same either way.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../../include/maise_b200.h"

int mb_handle_fail(int code, const char *msg);

static int cmp_int(const void *a, const void *b) { return *(const int *)a - *(const int *)b; }

int mb_parse_efile(mb_potential *pot, const char *dir, int index, int EFS, int N, int NM, int ND, int XT,
                   const int *atmn, const double *lat9, const double *x, double E, double p, double DE,
                   const int *marked, const double *frc_ref, const double *str_ref, const char *data_path) {
    char path[1200];
    FILE *f = NULL;
    int nspc, D, rc, i, n, q, NF = 0, DNmax = 0;
    double *G = NULL, *dG = NULL, *dx = NULL, *Sn = NULL, *blk = NULL;
    int *nn = NULL, *nj = NULL, *sh = NULL, *owners = NULL, *nown = NULL;
    if (!pot || !dir || index < 0 || EFS < 0 || EFS > 3 || N < 1 || !atmn || !lat9 || !x)
        return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    if ((rc = mb_model_info(pot, &nspc, NULL, &D, NULL))) return rc;
    G = (double *)malloc(sizeof(double) * (size_t)N * D);
    dG = (double *)malloc(sizeof(double) * (size_t)N * D);
    dx = (double *)calloc(3 * (size_t)N, sizeof(double));
    if (!G || !dG || !dx) { rc = mb_handle_fail(MB_ERR_ARG, "out of memory"); goto out; }
    if ((rc = mb_descriptors(pot, N, NM, ND, XT, atmn, lat9, x, G))) goto out;
    if (EFS == 1 || EFS == 3) {
        nn = (int *)malloc(sizeof(int) * N);
        nj = (int *)malloc(sizeof(int) * (size_t)N * NM);
        sh = (int *)malloc(sizeof(int) * 3 * (size_t)N * NM);
        owners = (int *)malloc(sizeof(int) * (size_t)N * NM);
        nown = (int *)calloc(N, sizeof(int));
        blk = (double *)malloc(sizeof(double) * 3 * (size_t)N * D); /* [atom][n][q] of one marked atom */
        if (!nn || !nj || !sh || !owners || !nown || !blk) { rc = mb_handle_fail(MB_ERR_ARG, "out of memory"); goto out; }
        if ((rc = mb_neighbours(pot, N, NM, ND, XT, atmn, lat9, x, 0, NM, nn, nj, sh, NULL))) goto out;
        for (i = 0; i < N; i++) {
            if (!marked || !marked[i]) continue;
            int k = 0, t;
            NF++;
            for (t = 0; t < nn[i]; t++) {
                const int j = nj[(size_t)i * NM + t];
                if (j != i) owners[(size_t)i * NM + k++] = j;
            }
            qsort(owners + (size_t)i * NM, k, sizeof(int), cmp_int);
            /* unique neighbour atoms (images of one atom count once) */
            {
                int u = 0;
                for (t = 0; t < k; t++)
                    if (t == 0 || owners[(size_t)i * NM + t] != owners[(size_t)i * NM + t - 1])
                        owners[(size_t)i * NM + u++] = owners[(size_t)i * NM + t];
                nown[i] = u;
            }
            if (nown[i] > DNmax) DNmax = nown[i];
        }
    }
    snprintf(path, sizeof(path), "%s/e%06d", dir, index);
    if (!(f = fopen(path, "w"))) { rc = mb_handle_fail(MB_ERR_ARG, "cannot write the descriptor file"); goto out; }
    fprintf(f, "%d %3d %3d %3d %3d   % lf  % lf  % lf\n", EFS, D, N, NF, DNmax, E, p, DE);
    if (EFS == 1 || EFS == 3) {
        for (i = 0; i < N; i++)
            if (marked && marked[i]) fprintf(f, "%3d ", i);
        fprintf(f, "\n");
    }
    if (EFS == 2 || EFS == 3) {
        for (q = 0; q < 6; q++) fprintf(f, "% 28.16lf ", str_ref ? str_ref[q] : 0.0);
        fprintf(f, "\n");
    }
    fprintf(f, "%s\n", data_path && data_path[0] ? data_path : "./");
    for (i = 0; i < N; i++) {
        fprintf(f, "%d\n", atmn[i]);
        for (n = 0; n < D; n++) fprintf(f, "% 28.16lf\n", G[(size_t)i * D + n]);
    }
    if (EFS == 1 || EFS == 3)
        for (i = 0; i < N; i++) {
            int t;
            if (!marked || !marked[i]) continue;
            for (q = 0; q < 3; q++) {
                memset(dx, 0, sizeof(double) * 3 * N);
                dx[3 * i + q] = 1.0;
                if ((rc = mb_descriptor_jvp(pot, N, NM, ND, XT, atmn, lat9, x, dx, NULL, dG))) goto out;
                for (t = 0; t < N * D; t++) blk[(size_t)t * 3 + q] = dG[t];
            }
            fprintf(f, "%4d %4d ", i, nown[i]);
            for (q = 0; q < 3; q++) fprintf(f, "% lf ", frc_ref ? frc_ref[3 * i + q] : 0.0);
            fprintf(f, "\n");
            for (n = 0; n < D; n++) {
                const double *b = blk + ((size_t)i * D + n) * 3;
                fprintf(f, "% 28.16lf % 28.16lf % 28.16lf\n", b[0], b[1], b[2]);
            }
            for (t = 0; t < nown[i]; t++) {
                const int j = owners[(size_t)i * NM + t];
                fprintf(f, "%4d\n", j);
                for (n = 0; n < D; n++) {
                    const double *b = blk + ((size_t)j * D + n) * 3;
                    fprintf(f, "% 28.16lf % 28.16lf % 28.16lf\n", b[0], b[1], b[2]);
                }
            }
        }
    if (EFS == 2 || EFS == 3) {
        /* strain columns in the virial's order: (q, (q+1) % 3) off the diagonal */
        static const int ab[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {1, 2}, {2, 0}};
        int k;
        Sn = (double *)malloc(sizeof(double) * 6 * (size_t)N * D);
        if (!Sn) { rc = mb_handle_fail(MB_ERR_ARG, "out of memory"); goto out; }
        for (k = 0; k < 6; k++) {
            double eps[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            eps[3 * ab[k][0] + ab[k][1]] = 1.0;
            if ((rc = mb_descriptor_jvp(pot, N, NM, ND, XT, atmn, lat9, x, NULL, eps, dG))) goto out;
            for (i = 0; i < N * D; i++) Sn[(size_t)i * 6 + k] = dG[i];
        }
        for (i = 0; i < N; i++)
            for (n = 0; n < D; n++) {
                for (k = 0; k < 6; k++) fprintf(f, "% 28.16lf ", Sn[((size_t)i * D + n) * 6 + k]);
                fprintf(f, "\n");
            }
    }
    rc = MB_OK;
out:
    if (f && fclose(f) && rc == MB_OK) rc = mb_handle_fail(MB_ERR_ARG, "cannot write the descriptor file");
    free(G); free(dG); free(dx); free(Sn); free(blk);
    free(nn); free(nj); free(sh); free(owners); free(nown);
    return rc;
}
