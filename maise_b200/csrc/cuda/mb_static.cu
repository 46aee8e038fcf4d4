/*
 * mb_static.cu -- energy/forces/virial of one structure without any device
 * allocation (mb_efs_noalloc, declared in include/maise_b200.h).
 *
 * Who needs it: host codes that own every byte of device memory themselves
 * -- an MD engine or a search driver that carves all of its buffers out of
 * one pre-sized pool, or runs under a fixed memory budget -- and so cannot
 * let a library call cudaMalloc in the middle of their time-step loop (an
 * allocation there can exceed their budget and makes the device
 * synchronise, which breaks the stream ordering they rely on).  They hand
 * in device pointers for the inputs and outputs; every intermediate (the
 * wrapped positions, the cell and neighbour lists, per-atom energies and
 * virials, status words) lives in the fixed array below.
 *
 * Limits: at most MB_STATIC_MAX_ATOMS atoms, MB_STATIC_MAX_NEIGHBOURS
 * neighbours per atom and MB_STATIC_MAX_CELLS cell-list bins (beyond that
 * many bins the all-pairs neighbour search is used).  The array takes about
 * 7.3 MB of device memory on every GPU that loads the library, for as long
 * as the process lives.
 */
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include "../../../include/maise_b200.h"
#include "../mb_internal.h"

#define MB_STATIC_MAX_ATOMS 2048
#define MB_STATIC_MAX_NEIGHBOURS 96
#define MB_STATIC_MAX_CELLS 4096

/* sizes of the scratch segments, each rounded up to 256 bytes */
#define SEG(bytes) ((((size_t)(bytes)) + 255) & ~(size_t)255)
#define S_X SEG(sizeof(double) * 3 * MB_STATIC_MAX_ATOMS)
#define S_NN SEG(sizeof(int) * MB_STATIC_MAX_ATOMS)
#define S_NJ SEG(sizeof(int) * MB_STATIC_MAX_ATOMS * MB_STATIC_MAX_NEIGHBOURS)
#define S_ND SEG(sizeof(double) * 4 * MB_STATIC_MAX_ATOMS * MB_STATIC_MAX_NEIGHBOURS)
#define S_EA SEG(sizeof(double) * MB_STATIC_MAX_ATOMS)
#define S_VIR SEG(sizeof(double) * 6 * MB_STATIC_MAX_ATOMS)
#define S_CELL SEG(sizeof(int) * MB_STATIC_MAX_ATOMS)
#define S_CCNT SEG(sizeof(int) * (MB_STATIC_MAX_CELLS + 1))
#define S_STAT SEG(sizeof(int) * 4 + sizeof(unsigned long long) * 2)
#define MB_STATIC_BYTES (S_X + S_NN + S_NJ + S_ND + 2 * S_EA + S_VIR + 2 * S_CELL + 2 * S_CCNT + S_STAT)

/* The scratch shared by every call on this device.  Host code must not
 * pass this symbol to a kernel: its device address is obtained once per
 * device with cudaGetSymbolAddress. */
static __device__ __align__(256) unsigned char mb_static_scratch[MB_STATIC_BYTES];

extern "C" {
const mb_model *mb_handle_model(const mb_potential *p);
int mb_handle_device(const mb_potential *p);
int mb_handle_fail(int code, const char *msg);
void mb_handle_geometry(const mb_potential *p, const double *lat9, int ND, int N, double p_gpa, mb_cell *c,
                        double *pV);
mb_params *mb_handle_dev_params(mb_potential *p);
double *mb_handle_dev_weights(mb_potential *p);
}

#define MB_MAX_DEVICES 64
static unsigned char *mb_static_base[MB_MAX_DEVICES];

/* device address of the scratch array on `dev` (the current device);
 * looked up on the first call on that device */
static unsigned char *static_base(int dev) {
    if (dev < 0 || dev >= MB_MAX_DEVICES) return nullptr;
    if (!mb_static_base[dev]) {
        void *ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, mb_static_scratch) != cudaSuccess) return nullptr;
        mb_static_base[dev] = (unsigned char *)ptr;
    }
    return mb_static_base[dev];
}

extern "C" int mb_efs_noalloc(mb_potential *pot, int N, int NM, int ND, const double *lat9, const double *d_x,
                              const int *d_spc, double p_gpa, double urep, double *d_frc, double *d_out,
                              void *stream) {
    if (!pot || !lat9 || !d_x || !d_spc || !d_frc || !d_out || NM < 1 || ND < 0 || ND > 3)
        return mb_handle_fail(MB_ERR_ARG, "bad arguments");
    if (N < 1 || N > MB_STATIC_MAX_ATOMS)
        return mb_handle_fail(MB_ERR_CAPACITY, "mb_efs_noalloc takes 1..2048 atoms (its fixed scratch size)");
    const int dev = mb_handle_device(pot);
    if (cudaSetDevice(dev) != cudaSuccess) return mb_handle_fail(MB_ERR_CUDA, "cudaSetDevice failed");
    unsigned char *base = static_base(dev);
    if (!base) return mb_handle_fail(MB_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
    cudaStream_t st = (cudaStream_t)stream;
    const mb_model *m = mb_handle_model(pot);

    mb_cell c;
    double pV = 0.0;
    mb_handle_geometry(pot, lat9, ND, N, p_gpa, &c, &pV);
    if (c.M[0] && (long)c.M[0] * c.M[1] * c.M[2] > MB_STATIC_MAX_CELLS) c.M[0] = c.M[1] = c.M[2] = 0;

    /* a working set pointing into the scratch array */
    mb_dev d;
    memset(&d, 0, sizeof(d));
    unsigned char *p = base;
    d.X = (double *)p; p += S_X;
    d.nn = (int *)p; p += S_NN;
    d.nj = (int *)p; p += S_NJ;
    d.nd = (double *)p; p += S_ND;
    d.EA = (double *)p; p += S_EA;
    d.EU = (double *)p; p += S_EA;
    d.vir = (double *)p; p += S_VIR;
    d.cell_of = (int *)p; p += S_CELL;
    d.cell_atoms = (int *)p; p += S_CELL;
    d.cell_cnt = (int *)p; p += S_CCNT;
    d.cell_start = (int *)p; p += S_CCNT;
    d.status = (int *)p;
    d.counters = (unsigned long long *)(p + 16);
    d.capN = MB_STATIC_MAX_ATOMS;
    d.capNB = MB_STATIC_MAX_NEIGHBOURS;
    d.capCells = MB_STATIC_MAX_CELLS;
    d.spc = (int *)d_spc;
    d.F = d_frc;
    d.out = d_out;
    d.params = mb_handle_dev_params(pot);
    d.weights = mb_handle_dev_weights(pot);
    d.tune_fixed = N >= 256 ? 0 : (N >= 64 ? 1 : 2);

    long launches = 0;
    int r;
    /* everything that must start at zero is cleared on the stream first */
    if (cudaMemcpyAsync(d.X, d_x, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(d.status, 0, sizeof(int) * 4 + sizeof(unsigned long long) * 2, st) != cudaSuccess)
        return mb_handle_fail(MB_ERR_CUDA, "staging the positions failed");
    const char *stage = "wrap";
    if (!(r = mbk_wrap(&d, N, &c, st, &launches)) && (stage = "neighbour list") &&
        !(r = mbk_nlist(&d, N, NM, &c, m->rc_list, st, &launches)) && (stage = "descriptor kernel") &&
        !(r = mbk_descriptor_pass(&d, m, N, MB_MODE_EFS, urep > 0.0 ? urep : 0.0, 0, 0, st, &launches)) &&
        (stage = "finalize"))
        r = mbk_finalize(&d, N, MB_MODE_EFS, pV, st, &launches);
    if (r) {
        static char msg[160];
        snprintf(msg, sizeof(msg), "%s: %s", stage, cudaGetErrorString((cudaError_t)r));
        return mb_handle_fail(MB_ERR_CUDA, msg);
    }
    int status[4] = {0, 0, 0, 0};
    if (cudaMemcpyAsync(status, d.status, sizeof(status), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return mb_handle_fail(MB_ERR_CUDA, "reading the status word failed");
    if (status[0] & MB_ST_WRAP) return mb_handle_fail(MB_ERR_STATE, "non-finite or runaway positions");
    if (status[0] & MB_ST_NBR_OVERFLOW) return mb_handle_fail(MB_ERR_NEIGHBOURS, "an atom reached NM neighbours");
    if (status[0] & MB_ST_CAP_OVERFLOW)
        return mb_handle_fail(MB_ERR_CAPACITY, "an atom has more than 96 neighbours (the fixed scratch size)");
    return MB_OK;
}
