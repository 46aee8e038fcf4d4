/*
 * maise_call.h -- drop-in for libmaise's energy/force/stress entry point
 *
 *   double CALL_MAISE(ANN *R, PRS *P, PRS *W, LNK *L, Cell *C, int CODE,
 *                     int N, int NM, int ND, int NP, int XT, int *ATMN,
 *                     double *LAT, double *X, double *FRC, double *STR);
 *
 * (reference: src/cmod.c:1136-1224; callers interface/c/c2maise.c:63,
 * interface/cpp/cpp2maise.cpp:66, interface/f90/maise.f90:9-23).
 *
 * Programs written for the reference include its mlib.h, which defines the
 * structures and declares CALL_MAISE; they relink against libmaise_b200
 * unchanged.  New C code may include this header instead: it provides
 * storage types of the reference's sizes.
 *
 * The structures are caller-owned storage.  As in the reference, L->B must
 * be 0 before the first call, which then reads ./model from the working
 * directory; C->p (pressure in GPa) is divided by eV2GPa in place on every
 * call; R->UREP (eV) enables the short-range repulsion when positive.  On
 * return C->E and C->H hold the energy and enthalpy.  No other field is
 * read or written.  NP (OpenMP threads) and CODE are ignored; the CUDA
 * device is taken from the environment variable MAISE_B200_DEVICE
 * (default 0).  Errors print a message to stderr and exit(1), as the
 * reference does; with MAISE_B200_NO_EXIT set, CALL_MAISE returns NaN
 * instead and mb_last_error() holds the message.
 */
#ifndef MAISE_CALL_H
#define MAISE_CALL_H

/* Byte sizes and field offsets of the reference's structures under the
 * x86-64 System V ABI (inc/cdef.h:9-135, inc/ndef.h:4-175).  Checked by
 * tests against the reference headers. */
#define MB_SIZEOF_ANN 4704
#define MB_SIZEOF_PRS 160
#define MB_SIZEOF_LNK 376
#define MB_SIZEOF_CELL 10624
#define MB_OFFSET_ANN_UREP 4688
#define MB_OFFSET_LNK_B 152
#define MB_OFFSET_CELL_P 1736
#define MB_OFFSET_CELL_E 2032
#define MB_OFFSET_CELL_H 1768

#ifndef MAISE /* the reference's mlib.h has not declared them */
typedef union { double align_; unsigned char bytes[MB_SIZEOF_ANN]; } ANN;
typedef union { double align_; unsigned char bytes[MB_SIZEOF_PRS]; } PRS;
typedef union { double align_; unsigned char bytes[MB_SIZEOF_LNK]; } LNK;
typedef union { double align_; unsigned char bytes[MB_SIZEOF_CELL]; } Cell;

#ifdef __cplusplus
extern "C" {
#endif
double CALL_MAISE(ANN *R, PRS *P, PRS *W, LNK *L, Cell *C, int CODE, int N, int NM, int ND, int NP, int XT, int *ATMN,
                  double *LAT, double *X, double *FRC, double *STR);
#ifdef __cplusplus
}
#endif
#endif

#endif
