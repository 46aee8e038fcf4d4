/*
 * mb_call_maise.c -- CALL_MAISE with the reference's signature and
 * semantics (src/cmod.c:1164-1224), backed by an mb_potential per LNK
 * object.  See include/maise_call.h for the contract.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../../include/maise_b200.h"
#include "../../../include/maise_call.h"

#define MB_EV2GPA 160.2176565 /* src/util.c:8 */
#define MB_MAX_LINKS 64

static struct {
    const void *L;
    mb_potential *pot;
} mb_links[MB_MAX_LINKS];

static double call_error(const char *what) {
    fprintf(stderr, "CALL_MAISE: %s: %s\n", what, mb_last_error());
    if (!getenv("MAISE_B200_NO_EXIT")) exit(1);
    return NAN;
}

static mb_potential *link_of(const void *L) {
    int k;
    for (k = 0; k < MB_MAX_LINKS; k++)
        if (mb_links[k].L == L) return mb_links[k].pot;
    return NULL;
}

double CALL_MAISE(ANN *R, PRS *P, PRS *W, LNK *L, Cell *C, int CODE, int N, int NM, int ND, int NP, int XT, int *ATMN,
                  double *LAT, double *X, double *FRC, double *STR) {
    int *built = (int *)((unsigned char *)L + MB_OFFSET_LNK_B);
    double *pres = (double *)((unsigned char *)C + MB_OFFSET_CELL_P);
    double urep = *(const double *)((const unsigned char *)R + MB_OFFSET_ANN_UREP);
    double p_gpa, H = 0.0, E = 0.0;
    mb_potential *pot;
    int rc;
    (void)P; (void)W; (void)CODE; (void)NP;
    /* the reference converts the pressure in place on every call (src/cmod.c:1181) */
    p_gpa = *pres;
    *pres = p_gpa / MB_EV2GPA;
    pot = link_of(L);
    if (*built == 0 || !pot) {
        const char *dev = getenv("MAISE_B200_DEVICE");
        int k;
        if (pot) {
            mb_close(pot);
            for (k = 0; k < MB_MAX_LINKS; k++)
                if (mb_links[k].L == L) mb_links[k].L = NULL;
        }
        rc = mb_open("model", dev ? atoi(dev) : 0, &pot);
        if (rc) return call_error("loading ./model");
        for (k = 0; k < MB_MAX_LINKS && mb_links[k].L; k++)
            ;
        if (k == MB_MAX_LINKS) return call_error("too many LNK objects");
        mb_links[k].L = L;
        mb_links[k].pot = pot;
        rc = mb_reserve(pot, N, NM < 64 ? NM : 64);
        if (rc) return call_error("reserving device memory");
        *built = 1;
    }
    if (!(urep > 0.0)) urep = 0.0;
    rc = mb_efs(pot, N, NM, ND, XT, ATMN, LAT, X, p_gpa, urep, &H, &E, FRC, STR, NULL, NULL);
    if (rc) return call_error("energy/force/stress evaluation");
    *(double *)((unsigned char *)C + MB_OFFSET_CELL_E) = E;
    *(double *)((unsigned char *)C + MB_OFFSET_CELL_H) = H;
    return H;
}
