/*
 * mb_core.c -- host side of libmaise_b200: handles, device memory, the
 * energy/force/stress call sequence, and the relax and NVT drivers.
 *
 * One call of mb_efs performs, on the handle's stream:
 *   H2D positions/species -> wrap (JAR) -> neighbour list (LIST) ->
 *   fused descriptor + MLP + force kernel -> finalize -> D2H results,
 * the sequence CELL_FRC runs on the CPU (src/cmod.c:153-191).
 */
#include <cuda_runtime_api.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../../include/maise_b200.h"
#include "../mb_internal.h"
#include "mb_bfgs.h"

#define MB_EV2GPA 160.2176565       /* src/util.c:8 */
#define MB_KB_INV 11604.0           /* K per eV, src/cmod.c:5 */
#define MB_PI 3.1415926535897932384626433832795

/* what an MD chunk graph was captured for: it is replayed only while all
 * of this is unchanged (buffers, sizes, step parameters, profiling state) */
typedef struct {
    long gen;
    int N, NM, chunk, st_on, ev_on, legs;
    double urep, dt, tau, T;
    mb_cell c;
    void *flush, *trace, *st_pool, *ev_pool;
    size_t flush_bytes;
} md_key;

/* what a single-structure pass graph was captured for */
typedef struct {
    long gen;
    int N, NM, ND, mode, M[3], legs;
    double urep;
    void *h_res;
} pass_key;

#define MB_PASS_NODES 8

typedef struct {
    cudaGraph_t g;
    cudaGraphExec_t x;
    pass_key k;
    void *nodes[MB_PASS_NODES];
    int rows[MB_PASS_NODES], count;
    long launches;
    mb_cell last_c;
    double last_pv;
    pass_key seen; /* last key run without a graph: captured when it repeats */
    int seen_valid;
} pass_graph;

struct mb_potential {
    mb_model m;
    int device;
    long long batch_evals, batch_work[3];
    float batch_ms;
    cudaStream_t stream;
    mb_dev d;
    long launches;
    long gen; /* advanced whenever device buffers are reallocated */
    /* host staging (pinned) */
    double *h_buf;
    size_t h_buf_len;
    int *h_status;
    double *h_out;
    /* leg tables for the descriptor pass: the model qualifies and they are
     * not switched off (MAISE_B200_LEGS=0) */
    int legs_enabled;
    /* MD chunk graph */
    int use_graphs;
    cudaGraphExec_t md_exec;
    md_key md_k;
    long md_launches;
    int md_st_events, md_ev_events;
    /* single-structure pass graphs, one per mode (a relax alternates energy
     * and energy+force passes): cell-dependent kernel nodes are re-pointed
     * at each call's cell; results staged in pinned h_res */
    pass_graph pgs[4];
    int pbroken;
    double *h_res; /* F[3N] then X[3N] of the last graphed pass */
    size_t h_res_len;
    int res_staged;
    /* timings moved out of the event pools (graph replays reuse the events) */
    double st_acc_ms, ev_acc_ms;
    int st_acc_n, ev_acc_n;
};

static __thread char mb_err[512];

const char *mb_last_error(void) { return mb_err; }

static int fail(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(mb_err, sizeof(mb_err), fmt, ap);
    va_end(ap);
    return code;
}

static int cuda_fail(cudaError_t e, const char *what) {
    return fail(MB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call, what)                              \
    do {                                            \
        cudaError_t e_ = (call);                    \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

/* ------------------------------------------------------------------ */
/* handle lifecycle                                                    */
/* ------------------------------------------------------------------ */

int mb_open(const char *model_path, int device, mb_potential **out) {
    mb_potential *p;
    struct cudaDeviceProp prop;
    int ndev = 0;
    char err[400];
    size_t wbytes;
    if (!model_path || !out) return fail(MB_ERR_ARG, "null argument");
    *out = NULL;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(MB_ERR_NOGPU, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(MB_ERR_ARG, "device %d out of range (%d devices)", device, ndev);
    CK(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    if (prop.major < 10) return fail(MB_ERR_NOGPU, "device %d is sm_%d%d; this build targets sm_100a", device, prop.major, prop.minor);
    p = (mb_potential *)calloc(1, sizeof(mb_potential));
    if (mb_model_load(model_path, &p->m, err, sizeof(err))) {
        free(p);
        return fail(MB_ERR_MODEL, "%s", err);
    }
    p->device = device;
    p->d.tune_fixed = -1;
    {
        const char *g = getenv("MAISE_B200_GRAPHS");
        p->use_graphs = !(g && g[0] == '0');
    }
    {
        const char *fx = getenv("MAISE_B200_SHAPE");
        if (fx) p->d.tune_fixed = atoi(fx);
    }
    {
        const char *lg = getenv("MAISE_B200_LEGS");
        p->legs_enabled = mbk_legs_model(&p->m) && !(lg && lg[0] == '0');
    }
    CK(cudaSetDevice(device), "cudaSetDevice");
    CK(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    CK(cudaMalloc((void **)&p->d.params, sizeof(mb_params)), "cudaMalloc params");
    CK(cudaMemcpy(p->d.params, &p->m.P, sizeof(mb_params), cudaMemcpyHostToDevice), "upload params");
    /* weights followed by the per-species masses (MD) */
    wbytes = sizeof(double) * (p->m.weights_len + MB_MAXSPC);
    CK(cudaMalloc((void **)&p->d.weights, wbytes), "cudaMalloc weights");
    CK(cudaMemcpy(p->d.weights, p->m.weights, sizeof(double) * p->m.weights_len, cudaMemcpyHostToDevice), "upload weights");
    CK(cudaMemcpy(p->d.weights + p->m.weights_len, p->m.mass, sizeof(double) * MB_MAXSPC, cudaMemcpyHostToDevice),
       "upload masses");
    CK(cudaMalloc((void **)&p->d.out, sizeof(double) * 16), "cudaMalloc out");
    CK(cudaMemset(p->d.out, 0, sizeof(double) * 16), "memset out");
    CK(cudaMalloc((void **)&p->d.part, sizeof(double) * 2 * MB_RED_MAXB * 8), "cudaMalloc part");
    CK(cudaMalloc((void **)&p->d.ticket, sizeof(unsigned) * 2), "cudaMalloc ticket");
    CK(cudaMemset(p->d.ticket, 0, sizeof(unsigned) * 2), "memset ticket");
    CK(cudaMalloc((void **)&p->d.status, sizeof(int) * 4), "cudaMalloc status");
    CK(cudaMalloc((void **)&p->d.counters, sizeof(unsigned long long) * 2), "cudaMalloc counters");
    CK(cudaMemset(p->d.counters, 0, sizeof(unsigned long long) * 2), "memset counters");
    CK(cudaMallocHost((void **)&p->h_status, sizeof(int) * 4), "cudaMallocHost");
    CK(cudaMallocHost((void **)&p->h_out, sizeof(double) * 16), "cudaMallocHost");
    *out = p;
    mb_err[0] = '\0';
    return MB_OK;
}

static void dev_free(mb_dev *d) {
    cudaFree(d->nk); cudaFree(d->leg); cudaFree(d->nso); cudaFree(d->trip); cudaFree(d->tboff); cudaFree(d->lhash);
    cudaFree(d->X); cudaFree(d->V); cudaFree(d->spc); cudaFree(d->nn); cudaFree(d->nj); cudaFree(d->nd);
    cudaFree(d->F); cudaFree(d->EA); cudaFree(d->EU); cudaFree(d->vir); cudaFree(d->G);
    cudaFree(d->cell_of); cudaFree(d->cell_cnt); cudaFree(d->cell_start); cudaFree(d->cell_atoms);
    cudaFree(d->trace);
}

int mb_close(mb_potential *p) {
    if (!p) return MB_OK;
    cudaSetDevice(p->device);
    cudaStreamSynchronize(p->stream);
    if (p->md_exec) cudaGraphExecDestroy(p->md_exec);
    {
        int k;
        for (k = 0; k < 4; k++) {
            if (p->pgs[k].x) cudaGraphExecDestroy(p->pgs[k].x);
            if (p->pgs[k].g) cudaGraphDestroy(p->pgs[k].g);
        }
    }
    cudaFreeHost(p->h_res);
    dev_free(&p->d);
    cudaFree(p->d.params);
    cudaFree(p->d.weights);
    cudaFree(p->d.out);
    cudaFree(p->d.part);
    cudaFree(p->d.ticket);
    cudaFree(p->d.status);
    cudaFree(p->d.counters);
    cudaFree(p->d.flush);
    if (p->d.st_pool) {
        int k;
        for (k = 0; k < 2 * p->d.st_cap; k++) cudaEventDestroy(((cudaEvent_t *)p->d.st_pool)[k]);
        free(p->d.st_pool);
    }
    if (p->d.ev_pool) {
        int k;
        for (k = 0; k < 2 * p->d.ev_cap; k++) cudaEventDestroy(((cudaEvent_t *)p->d.ev_pool)[k]);
        free(p->d.ev_pool);
    }
    cudaFreeHost(p->h_status);
    cudaFreeHost(p->h_out);
    cudaFreeHost(p->h_buf);
    cudaStreamDestroy(p->stream);
    mb_model_free(&p->m);
    free(p);
    return MB_OK;
}

int mb_model_info(const mb_potential *p, int *nspc, int *spcz, int *D, double *rc) {
    int s;
    if (!p) return fail(MB_ERR_ARG, "null handle");
    if (nspc) *nspc = p->m.nspc;
    if (spcz)
        for (s = 0; s < p->m.nspc; s++) spcz[s] = p->m.spcz[s];
    if (D) *D = p->m.P.D;
    if (rc) *rc = p->m.rc_list;
    return MB_OK;
}

void *mb_stream(mb_potential *p) { return p ? (void *)p->stream : NULL; }

/* accessors for the other host files (mb_batch.c) */
const mb_model *mb_handle_model(const mb_potential *p) { return &p->m; }
void *mb_handle_stream(mb_potential *p) { return (void *)p->stream; }
int mb_handle_device(const mb_potential *p) { return p->device; }
int mb_handle_fail(int code, const char *msg) { return fail(code, "%s", msg); }
void mb_handle_set_batch_stats(mb_potential *p, const long long *evals, float ms) {
    p->batch_evals = evals[0];
    p->batch_work[0] = evals[1];
    p->batch_work[1] = evals[2];
    p->batch_work[2] = evals[3];
    p->batch_ms = ms;
}

int mb_batch_stats(const mb_potential *p, long long *evals, double *ms) {
    if (!p) return fail(MB_ERR_ARG, "null handle");
    if (evals) *evals = p->batch_evals;
    if (ms) *ms = p->batch_ms;
    return MB_OK;
}

int mb_tune_read(const mb_potential *p, int cap, int *count, int *mode, int *legs, int *size_bucket, int *capacity,
                 int *wpa, int *apb, int *layout) {
    int k, n;
    if (!p || cap < 0 || !count) return fail(MB_ERR_ARG, "bad arguments");
    n = p->d.tune_n < cap ? p->d.tune_n : cap;
    *count = n;
    for (k = 0; k < n; k++) {
        /* a key with the leg path usable holds 16 + shape when the leg kernel
         * won and a k_efs shape otherwise */
        const int key = p->d.tune_key[k], v = p->d.tune_val[k], lg = ((key >> 26) & 1) && v >= 16;
        mode[k] = key >> 28;
        legs[k] = lg;
        size_bucket[k] = (key >> 20) & 0x3f;
        capacity[k] = key & 0xfffff;
        if (mbk_shape_dims(lg, lg ? v - 16 : v, &wpa[k], &apb[k])) wpa[k] = apb[k] = 0;
        layout[k] = lg && v - 16 >= 4; /* leg shapes 4-7: reverse pass over consecutive entries */
    }
    return MB_OK;
}

int mb_batch_work(const mb_potential *p, long long *atom_evals, long long *pairs, long long *triplets) {
    if (!p) return fail(MB_ERR_ARG, "null handle");
    if (atom_evals) *atom_evals = p->batch_work[0];
    if (pairs) *pairs = p->batch_work[1];
    if (triplets) *triplets = p->batch_work[2];
    return MB_OK;
}

int mb_profile(mb_potential *p, int enable, int capacity) {
    mb_dev *d;
    int k;
    if (!p) return fail(MB_ERR_ARG, "null handle");
    d = &p->d;
    CK(cudaSetDevice(p->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(p->stream), "synchronize");
    if (enable && capacity > d->ev_cap) {
        cudaEvent_t *pool;
        if (d->ev_pool) {
            for (k = 0; k < 2 * d->ev_cap; k++) cudaEventDestroy(((cudaEvent_t *)d->ev_pool)[k]);
            free(d->ev_pool);
        }
        pool = (cudaEvent_t *)calloc(2 * (size_t)capacity, sizeof(cudaEvent_t));
        for (k = 0; k < 2 * capacity; k++) CK(cudaEventCreate(&pool[k]), "cudaEventCreate");
        d->ev_pool = pool;
        d->ev_cap = capacity;
    }
    d->ev_on = enable ? 1 : 0;
    d->ev_n = 0;
    p->ev_acc_ms = 0.0;
    p->ev_acc_n = 0;
    CK(cudaMemsetAsync(d->counters, 0, sizeof(unsigned long long) * 2, p->stream), "memset counters");
    CK(cudaStreamSynchronize(p->stream), "synchronize");
    return MB_OK;
}

int mb_md_profile(mb_potential *p, int enable, int capacity, size_t flush_bytes) {
    mb_dev *d;
    int k;
    if (!p) return fail(MB_ERR_ARG, "null handle");
    d = &p->d;
    CK(cudaSetDevice(p->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(p->stream), "synchronize");
    if (enable && capacity > d->st_cap) {
        cudaEvent_t *pool;
        if (d->st_pool) {
            for (k = 0; k < 2 * d->st_cap; k++) cudaEventDestroy(((cudaEvent_t *)d->st_pool)[k]);
            free(d->st_pool);
        }
        pool = (cudaEvent_t *)calloc(2 * (size_t)capacity, sizeof(cudaEvent_t));
        for (k = 0; k < 2 * capacity; k++) CK(cudaEventCreate(&pool[k]), "cudaEventCreate");
        d->st_pool = pool;
        d->st_cap = capacity;
    }
    if (enable && flush_bytes > d->flush_bytes) {
        cudaFree(d->flush);
        d->flush = NULL;
        CK(cudaMalloc(&d->flush, flush_bytes), "alloc flush buffer");
    }
    if (enable) d->flush_bytes = flush_bytes > d->flush_bytes ? flush_bytes : d->flush_bytes;
    d->st_on = enable ? 1 : 0;
    d->st_n = 0;
    p->st_acc_ms = 0.0;
    p->st_acc_n = 0;
    return MB_OK;
}

int mb_md_profile_read(mb_potential *p, double *total_ms, int *steps) {
    double tot = 0.0;
    int k;
    if (!p) return fail(MB_ERR_ARG, "null handle");
    CK(cudaSetDevice(p->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(p->stream), "synchronize");
    for (k = 0; k < p->d.st_n; k++) {
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, ((cudaEvent_t *)p->d.st_pool)[2 * k], ((cudaEvent_t *)p->d.st_pool)[2 * k + 1]),
           "cudaEventElapsedTime");
        tot += ms;
    }
    if (total_ms) *total_ms = tot + p->st_acc_ms;
    if (steps) *steps = p->d.st_n + p->st_acc_n;
    return MB_OK;
}

int mb_profile_read(mb_potential *p, double *total_ms, int *launches, unsigned long long *pairs,
                    unsigned long long *triplets) {
    unsigned long long c[2];
    double tot = 0.0;
    int k;
    if (!p) return fail(MB_ERR_ARG, "null handle");
    CK(cudaSetDevice(p->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(p->stream), "synchronize");
    for (k = 0; k < p->d.ev_n; k++) {
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, ((cudaEvent_t *)p->d.ev_pool)[2 * k], ((cudaEvent_t *)p->d.ev_pool)[2 * k + 1]),
           "cudaEventElapsedTime");
        tot += ms;
    }
    CK(cudaMemcpy(c, p->d.counters, sizeof(c), cudaMemcpyDeviceToHost), "D2H counters");
    if (total_ms) *total_ms = tot + p->ev_acc_ms;
    if (launches) *launches = p->d.ev_n + p->ev_acc_n;
    if (pairs) *pairs = c[0];
    if (triplets) *triplets = c[1];
    return MB_OK;
}
long mb_launch_count(const mb_potential *p) { return p ? p->launches : 0; }

int mb_graphs(mb_potential *p, int enable) {
    if (!p) return fail(MB_ERR_ARG, "null handle");
    p->use_graphs = enable ? 1 : 0;
    return MB_OK;
}

/* grow device arrays to N atoms / nb neighbours per atom / ncell bins */
static int ensure(mb_potential *p, int N, int nb, int ncell) {
    mb_dev *d = &p->d;
    int D = p->m.P.D;
    if (N > d->capN) {
        int cap = N > 2 * d->capN ? N : 2 * d->capN;
        cudaFree(d->X); cudaFree(d->V); cudaFree(d->spc); cudaFree(d->nn); cudaFree(d->F); cudaFree(d->EA);
        cudaFree(d->EU); cudaFree(d->vir); cudaFree(d->G); cudaFree(d->cell_of); cudaFree(d->cell_atoms);
        CK(cudaMalloc((void **)&d->X, sizeof(double) * 3 * cap), "alloc X");
        CK(cudaMalloc((void **)&d->V, sizeof(double) * 3 * cap), "alloc V");
        CK(cudaMalloc((void **)&d->spc, sizeof(int) * cap), "alloc spc");
        CK(cudaMalloc((void **)&d->nn, sizeof(int) * cap), "alloc nn");
        CK(cudaMalloc((void **)&d->F, sizeof(double) * 3 * cap), "alloc F");
        CK(cudaMalloc((void **)&d->EA, sizeof(double) * cap), "alloc EA");
        CK(cudaMalloc((void **)&d->EU, sizeof(double) * cap), "alloc EU");
        CK(cudaMalloc((void **)&d->vir, sizeof(double) * 6 * cap), "alloc vir");
        CK(cudaMalloc((void **)&d->G, sizeof(double) * (size_t)D * cap), "alloc G");
        CK(cudaMalloc((void **)&d->cell_of, sizeof(int) * cap), "alloc cell_of");
        CK(cudaMalloc((void **)&d->cell_atoms, sizeof(int) * cap), "alloc cell_atoms");
        d->capN = cap;
        p->gen++;
        cudaFree(d->nj); cudaFree(d->nd); cudaFree(d->nk); cudaFree(d->leg); cudaFree(d->nso);
        cudaFree(d->trip); cudaFree(d->tboff); cudaFree(d->lhash);
        d->nj = NULL; d->nd = NULL; d->nk = NULL; d->leg = NULL; d->nso = NULL; d->trip = NULL; d->tboff = NULL;
        d->lhash = NULL;
        d->capNB = 0;
    }
    if (nb > d->capNB || !d->nj) {
        int cap = nb > d->capNB ? nb : d->capNB;
        cap = (cap + 7) & ~7;
        cudaFree(d->nj); cudaFree(d->nd); cudaFree(d->nk); cudaFree(d->leg); cudaFree(d->nso);
        cudaFree(d->trip); cudaFree(d->tboff); cudaFree(d->lhash);
        d->nk = NULL; d->leg = NULL; d->nso = NULL; d->trip = NULL; d->tboff = NULL; d->lhash = NULL;
        CK(cudaMalloc((void **)&d->nj, sizeof(int) * (size_t)cap * d->capN), "alloc nj");
        CK(cudaMalloc((void **)&d->nd, sizeof(double) * 4 * (size_t)cap * d->capN), "alloc nd");
        if (p->legs_enabled && cap <= MB_LEG_MAX_CAP) {
            /* leg tables of the descriptor pass (the model qualifies for them) */
            CK(cudaMalloc((void **)&d->nk, sizeof(unsigned) * (size_t)cap * d->capN), "alloc nk");
            CK(cudaMalloc((void **)&d->leg, sizeof(double) * MB_LEG_STRIDE * (size_t)cap * d->capN), "alloc legs");
            CK(cudaMalloc((void **)&d->nso, sizeof(int) * 4 * (size_t)d->capN), "alloc nso");
            d->tcap = cap * (cap - 1) / 2;
            CK(cudaMalloc((void **)&d->trip, 2 * sizeof(unsigned) * (size_t)d->tcap * d->capN), "alloc trip");
            CK(cudaMalloc((void **)&d->tboff, sizeof(int) * 8 * (size_t)d->capN), "alloc tboff");
            CK(cudaMalloc((void **)&d->lhash, 2 * sizeof(unsigned) * 256 * (size_t)d->capN), "alloc list hash");
        }
        d->capNB = cap;
        p->gen++;
    }
    if (ncell + 1 > d->capCells) {
        int cap = ncell + 1 > 2 * d->capCells ? ncell + 1 : 2 * d->capCells;
        cudaFree(d->cell_cnt); cudaFree(d->cell_start);
        CK(cudaMalloc((void **)&d->cell_cnt, sizeof(int) * cap), "alloc cell_cnt");
        CK(cudaMalloc((void **)&d->cell_start, sizeof(int) * (cap + 1)), "alloc cell_start");
        d->capCells = cap;
        p->gen++;
    }
    return MB_OK;
}

int mb_reserve(mb_potential *p, int max_atoms, int max_neighbours) {
    if (!p || max_atoms < 1 || max_neighbours < 1) return fail(MB_ERR_ARG, "bad reservation");
    CK(cudaSetDevice(p->device), "cudaSetDevice");
    return ensure(p, max_atoms, max_neighbours, 1);
}

static int host_buf(mb_potential *p, size_t n) {
    if (n <= p->h_buf_len) return MB_OK;
    cudaFreeHost(p->h_buf);
    p->h_buf = NULL;
    CK(cudaMallocHost((void **)&p->h_buf, sizeof(double) * n), "cudaMallocHost");
    p->h_buf_len = n;
    return MB_OK;
}

/* ------------------------------------------------------------------ */
/* geometry                                                            */
/* ------------------------------------------------------------------ */

/* reciprocal rows without 2 pi (Reciprocal, src/cell.c:432-443) */
static void reciprocal(const double *L, double *R) {
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

/* CELL_VOL for periodic cells (src/cutl.c:178-188) */
static double cell_volume(const double *L) {
    double V = L[0] * L[4] * L[8] + L[2] * L[3] * L[7] + L[1] * L[5] * L[6] - L[0] * L[5] * L[7] -
               L[1] * L[3] * L[8] - L[2] * L[4] * L[6];
    return fabs(V);
}

/* bins: 0 as the passes choose (cell list for N >= 64 when every periodic
 * direction holds >= 3 bins no thinner than Rc and there are >= 8 bins),
 * 1 never (all-pairs search), 2 whenever the bins are valid (periodic
 * directions >= 3 bins), whatever N */
static void setup_cell_bins(const mb_potential *p, const double *lat9, int ND, int N, mb_cell *c, int bins) {
    double rc = p->m.rc_list;
    int q;
    memset(c, 0, sizeof(*c));
    memcpy(c->L, lat9, sizeof(double) * 9);
    reciprocal(c->L, c->R);
    c->ND = ND;
    for (q = 0; q < 3; q++) {
        double len = sqrt(c->R[3 * q] * c->R[3 * q] + c->R[3 * q + 1] * c->R[3 * q + 1] + c->R[3 * q + 2] * c->R[3 * q + 2]);
        c->Nq[q] = q < ND ? (int)ceil(rc * len) : 0;
    }
    /* bins no thinner than Rc; periodic directions need at least 3 */
    if (bins != 1) {
        int M[3], ok = bins == 2 || N >= 64, total;
        for (q = 0; q < 3; q++) {
            double len = sqrt(c->R[3 * q] * c->R[3 * q] + c->R[3 * q + 1] * c->R[3 * q + 1] +
                              c->R[3 * q + 2] * c->R[3 * q + 2]);
            double w = rc * len * (1.0 + 1e-9) + 1e-12;
            double m = floor(1.0 / w);
            M[q] = m > 256.0 ? 256 : (int)m;
            if (M[q] < 1) M[q] = 1;
            if (q < ND && M[q] < 3) ok = 0;
        }
        total = M[0] * M[1] * M[2];
        if (ok && (bins == 2 || total >= 8))
            for (q = 0; q < 3; q++) c->M[q] = M[q];
    }
}

static void setup_cell(const mb_potential *p, const double *lat9, int ND, int N, mb_cell *c) {
    setup_cell_bins(p, lat9, ND, N, c, 0);
}

/* accessors used by mb_static.cu */
void mb_handle_geometry(const mb_potential *p, const double *lat9, int ND, int N, double p_gpa, mb_cell *c, double *pV) {
    setup_cell(p, lat9, ND, N, c);
    *pV = ND == 3 ? p_gpa / MB_EV2GPA * cell_volume(lat9) : 0.0;
}
mb_params *mb_handle_dev_params(mb_potential *p) { return p->d.params; }
double *mb_handle_dev_weights(mb_potential *p) { return p->d.weights; }

/* fractional -> Cartesian as CAST_CELL does (src/cmod.c:1108-1117) */
static void frac_to_cart(int N, const double *xf, const double *L, double *x) {
    int i, q, j;
    for (i = 0; i < N; i++)
        for (q = 0; q < 3; q++) {
            double s = 0.0;
            for (j = 0; j < 3; j++) s += xf[3 * i + j] * L[3 * j + q];
            x[3 * i + q] = s;
        }
}

/* ------------------------------------------------------------------ */
/* the E / E+F+S sequence                                              */
/* ------------------------------------------------------------------ */

static int upload(mb_potential *p, int N, int XT, const int *atmn, const double *lat9, const double *x) {
    int r, s;
    double *hx;
    for (s = 0; s < N; s++)
        if (atmn[s] < 0 || atmn[s] >= p->m.nspc) return fail(MB_ERR_ARG, "atom %d has species %d (model has %d)", s, atmn[s], p->m.nspc);
    if ((r = host_buf(p, 3 * (size_t)N + N))) return r;
    hx = p->h_buf;
    if (XT == 0)
        frac_to_cart(N, x, lat9, hx);
    else
        memcpy(hx, x, sizeof(double) * 3 * N);
    memcpy((int *)(hx + 3 * N), atmn, sizeof(int) * N);
    CK(cudaMemcpyAsync(p->d.X, hx, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, p->stream), "H2D positions");
    CK(cudaMemcpyAsync(p->d.spc, hx + 3 * N, sizeof(int) * N, cudaMemcpyHostToDevice, p->stream), "H2D species");
    return MB_OK;
}

/* Runs wrap -> list -> descriptor pass -> finalize once on the
 * device-resident positions and synchronises; h_out then holds E, H, U and
 * h_status the flags.  Returns MB_RETRY when the neighbour capacity had to
 * grow: the positions were already wrapped in place, so the caller
 * re-uploads them and calls again. */
#define MB_RETRY 1000
/* the device part of one pass, queued on the handle's stream: wrap, list,
 * descriptor pass, finalize, then the status word and E, H, U to the host
 * (and, with stage set, F and the wrapped X into the pinned h_res) */
static int enqueue_pass(mb_potential *p, int N, int NM, const mb_cell *c, double pV, int mode, double urep,
                        int stage) {
    int r;
    CK(cudaMemsetAsync(p->d.status, 0, sizeof(int) * 4, p->stream), "memset status");
    if ((r = mbk_wrap(&p->d, N, c, p->stream, &p->launches))) return cuda_fail((cudaError_t)r, "wrap");
    if ((r = mbk_nlist(&p->d, N, NM, c, p->m.rc_list, p->stream, &p->launches)))
        return cuda_fail((cudaError_t)r, "neighbour list");
    if ((r = mbk_descriptor_pass(&p->d, &p->m, N, mode, urep, 0, 0, p->stream, &p->launches)))
        return cuda_fail((cudaError_t)r, "descriptor kernel");
    if (mode != MB_MODE_DESCRIPTORS)
        if ((r = mbk_finalize(&p->d, N, mode, pV, p->stream, &p->launches))) return cuda_fail((cudaError_t)r, "finalize");
    CK(cudaMemcpyAsync(p->h_status, p->d.status, sizeof(int) * 4, cudaMemcpyDeviceToHost, p->stream), "D2H status");
    CK(cudaMemcpyAsync(p->h_out, p->d.out, sizeof(double) * 16, cudaMemcpyDeviceToHost, p->stream), "D2H out");
    if (stage) {
        if (mode == MB_MODE_EFS || mode == MB_MODE_VJP)
            CK(cudaMemcpyAsync(p->h_res, p->d.F, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, p->stream), "D2H F");
        CK(cudaMemcpyAsync(p->h_res + 3 * N, p->d.X, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, p->stream),
           "D2H X");
    }
    return MB_OK;
}

static void drop_pass_graph(pass_graph *q) {
    if (q->x) cudaGraphExecDestroy(q->x);
    if (q->g) cudaGraphDestroy(q->g);
    q->x = NULL;
    q->g = NULL;
}

/* Queue one pass as a replay of the captured pass graph of its mode,
 * capturing it first if nothing matches (MB_FALLBACK when a graph cannot be
 * used).  Between replays only the cell and pV change: the kernel nodes
 * that take them by value are re-pointed at the new values. */
#define MB_FALLBACK 1001
static int graph_pass(mb_potential *p, int N, int NM, int ND, const mb_cell *c, double pV, int mode, double urep) {
    pass_key k;
    pass_graph *q = &p->pgs[mode & 3];
    int r, m;
    if (6 * (size_t)N > p->h_res_len) {
        for (m = 0; m < 4; m++) drop_pass_graph(&p->pgs[m]);
        cudaFreeHost(p->h_res);
        p->h_res = NULL;
        p->h_res_len = 0;
        CK(cudaMallocHost((void **)&p->h_res, sizeof(double) * 6 * N), "cudaMallocHost");
        p->h_res_len = 6 * (size_t)N;
    }
    memset(&k, 0, sizeof(k));
    k.gen = p->gen;
    k.N = N;
    k.NM = NM;
    k.ND = ND;
    k.mode = mode;
    k.M[0] = c->M[0];
    k.M[1] = c->M[1];
    k.M[2] = c->M[2];
    k.urep = urep;
    k.h_res = p->h_res;
    k.legs = p->d.legs_on;
    if (!q->x || memcmp(&k, &q->k, sizeof(k))) {
        cudaGraph_t g = NULL;
        if (!q->seen_valid || memcmp(&k, &q->seen, sizeof(k))) {
            /* a key met once (e.g. a loop over structures of many sizes) is not
             * worth a capture: run it plainly and capture if it comes again */
            q->seen = k;
            q->seen_valid = 1;
            return MB_FALLBACK;
        }
        cudaError_t e;
        const long l0 = p->launches;
        const int expect = (ND > 0) + (c->M[0] > 0 ? 2 : 1) + (mode != MB_MODE_DESCRIPTORS);
        drop_pass_graph(q);
        CK(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        r = enqueue_pass(p, N, NM, c, pV, mode, urep, 1);
        e = cudaStreamEndCapture(p->stream, &g);
        if (r) {
            if (g) cudaGraphDestroy(g);
            return r;
        }
        if (e != cudaSuccess) return cuda_fail(e, "end capture");
        q->launches = p->launches - l0;
        p->launches = l0;
        q->count = mbk_graph_cell_nodes(g, q->nodes, q->rows, MB_PASS_NODES);
        if (q->count != expect) {
            /* the cell-dependent nodes were not all recognised: use plain launches */
            cudaGraphDestroy(g);
            p->pbroken = 1;
            return MB_FALLBACK;
        }
        e = cudaGraphInstantiate(&q->x, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            q->x = NULL;
            return cuda_fail(e, "graph instantiate");
        }
        q->g = g;
        q->k = k;
        q->last_c = *c;
        q->last_pv = pV;
    } else if (memcmp(c, &q->last_c, sizeof(*c)) || pV != q->last_pv) {
        if ((r = mbk_graph_set_cell(q->x, q->nodes, q->rows, q->count, c, pV)))
            return cuda_fail((cudaError_t)r, "graph node update");
        q->last_c = *c;
        q->last_pv = pV;
    }
    CK(cudaGraphLaunch(q->x, p->stream), "graph launch");
    p->launches += q->launches;
    p->res_staged = 1;
    return MB_OK;
}

static int run_pass(mb_potential *p, int N, int NM, int ND, const double *lat9, int mode, double urep, double p_gpa) {
    mb_cell c;
    double pV = 0.0;
    int r, ncell;
    setup_cell(p, lat9, ND, N, &c);
    if (ND == 3) pV = p_gpa / MB_EV2GPA * cell_volume(lat9);
    ncell = c.M[0] ? c.M[0] * c.M[1] * c.M[2] : 1;
    if ((r = ensure(p, N, p->d.capNB ? p->d.capNB : (NM < 64 ? NM : 64), ncell))) return r;
    p->d.legs_on = mbk_legs_usable(&p->d, &p->m, N, &c);
    p->res_staged = 0;
    r = MB_FALLBACK;
    if (p->use_graphs && !p->pbroken && !p->d.ev_on && mbk_shape_ready(&p->d, N, mode)) {
        r = graph_pass(p, N, NM, ND, &c, pV, mode, urep);
        if (r != MB_OK && r != MB_FALLBACK) return r;
    }
    if (r == MB_FALLBACK && (r = enqueue_pass(p, N, NM, &c, pV, mode, urep, 0))) return r;
    CK(cudaStreamSynchronize(p->stream), "synchronize");
    if (p->h_status[0] & MB_ST_WRAP) return fail(MB_ERR_STATE, "non-finite or runaway positions");
    if (p->h_status[0] & MB_ST_NBR_OVERFLOW)
        return fail(MB_ERR_NEIGHBOURS, "an atom reached NM=%d neighbours within %.4f A; increase NM", NM, p->m.rc_list);
    if (p->h_status[0] & MB_ST_CAP_OVERFLOW) {
        if ((r = ensure(p, N, p->h_status[1] + 8, ncell))) return r;
        return MB_RETRY;
    }
    return MB_OK;
}

/* host-array entry: upload then run, retrying with a fresh upload when the
 * neighbour capacity had to grow (the wrap is done in place on device) */
static int host_pass(mb_potential *p, int N, int NM, int ND, int XT, const int *atmn, const double *lat9,
                     const double *x, int mode, double urep, double p_gpa) {
    int r, tries;
    if (!p || N < 1 || NM < 1 || ND < 0 || ND > 3 || !atmn || !lat9 || !x) return fail(MB_ERR_ARG, "bad arguments");
    CK(cudaSetDevice(p->device), "cudaSetDevice");
    if ((r = ensure(p, N, p->d.capNB ? p->d.capNB : (NM < 64 ? NM : 64), 1))) return r;
    for (tries = 0; tries < 3; tries++) {
        if ((r = upload(p, N, XT, atmn, lat9, x))) return r;
        r = run_pass(p, N, NM, ND, lat9, mode, urep, p_gpa);
        if (r != MB_RETRY) return r;
    }
    return fail(MB_ERR_CAPACITY, "neighbour capacity could not be established");
}

int mb_efs(mb_potential *p, int N, int NM, int ND, int XT, const int *atmn, const double *lat9, const double *x,
           double p_gpa, double urep, double *H, double *E, double *frc, double *str, double *ea, double *x_wrapped) {
    int r = host_pass(p, N, NM, ND, XT, atmn, lat9, x, MB_MODE_EFS, urep, p_gpa), k;
    if (r) return r;
    if (H) *H = p->h_out[1];
    if (E) *E = p->h_out[0];
    if (str)
        for (k = 0; k < 6; k++) str[k] = p->h_out[2 + k];
    if (p->res_staged) {
        /* the replayed pass left F and the wrapped X in pinned staging */
        if (frc) memcpy(frc, p->h_res, sizeof(double) * 3 * N);
        if (x_wrapped) memcpy(x_wrapped, p->h_res + 3 * N, sizeof(double) * 3 * N);
        if (!ea) return MB_OK;
    } else {
        if (frc) CK(cudaMemcpyAsync(frc, p->d.F, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, p->stream), "D2H forces");
        if (x_wrapped)
            CK(cudaMemcpyAsync(x_wrapped, p->d.X, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, p->stream), "D2H X");
    }
    if (ea) CK(cudaMemcpyAsync(ea, p->d.EA, sizeof(double) * N, cudaMemcpyDeviceToHost, p->stream), "D2H EA");
    CK(cudaStreamSynchronize(p->stream), "synchronize");
    return MB_OK;
}

int mb_energy(mb_potential *p, int N, int NM, int ND, int XT, const int *atmn, const double *lat9, const double *x,
              double p_gpa, double urep, double *H, double *E, double *ea) {
    int r = host_pass(p, N, NM, ND, XT, atmn, lat9, x, MB_MODE_ENERGY, urep, p_gpa);
    if (r) return r;
    if (H) *H = p->h_out[1];
    if (E) *E = p->h_out[0];
    if (ea) {
        CK(cudaMemcpyAsync(ea, p->d.EA, sizeof(double) * N, cudaMemcpyDeviceToHost, p->stream), "D2H EA");
        CK(cudaStreamSynchronize(p->stream), "synchronize");
    }
    return MB_OK;
}

int mb_descriptors(mb_potential *p, int N, int NM, int ND, int XT, const int *atmn, const double *lat9,
                   const double *x, double *G) {
    int r = host_pass(p, N, NM, ND, XT, atmn, lat9, x, MB_MODE_DESCRIPTORS, 0.0, 0.0);
    if (r) return r;
    if (!G) return MB_OK;
    CK(cudaMemcpyAsync(G, p->d.G, sizeof(double) * (size_t)N * p->m.P.D, cudaMemcpyDeviceToHost, p->stream), "D2H G");
    CK(cudaStreamSynchronize(p->stream), "synchronize");
    return MB_OK;
}

int mb_descriptor_vjp(mb_potential *p, int N, int NM, int ND, int XT, const int *atmn, const double *lat9,
                      const double *x, const double *g, double *frc, double *str) {
    int r, k;
    if (!g) return fail(MB_ERR_ARG, "null weights");
    if (!p || N < 1) return fail(MB_ERR_ARG, "bad arguments");
    CK(cudaSetDevice(p->device), "cudaSetDevice");
    if ((r = ensure(p, N, p->d.capNB ? p->d.capNB : (NM < 64 ? NM : 64), 1))) return r;
    CK(cudaMemcpyAsync(p->d.G, g, sizeof(double) * (size_t)N * p->m.P.D, cudaMemcpyHostToDevice, p->stream), "H2D g");
    r = host_pass(p, N, NM, ND, XT, atmn, lat9, x, MB_MODE_VJP, 0.0, 0.0);
    if (r) return r;
    if (str)
        for (k = 0; k < 6; k++) str[k] = p->h_out[2 + k];
    if (frc) CK(cudaMemcpyAsync(frc, p->d.F, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, p->stream), "D2H forces");
    CK(cudaStreamSynchronize(p->stream), "synchronize");
    return MB_OK;
}

int mb_neighbours(mb_potential *p, int N, int NM, int ND, int XT, const int *atmn, const double *lat9, const double *x,
                  int path, int cap, int *nn, int *nj, int *shift, double *x_wrapped) {
    mb_cell c;
    int r, tries, i, t, q, ncell, capNB;
    int *hnn = NULL, *hnj = NULL;
    double *hnd = NULL, *hx = NULL;
    if (!p || N < 1 || NM < 1 || ND < 0 || ND > 3 || !atmn || !lat9 || !x || cap < 1 || !nn || !nj || !shift ||
        path < 0 || path > 2)
        return fail(MB_ERR_ARG, "bad arguments");
    CK(cudaSetDevice(p->device), "cudaSetDevice");
    setup_cell_bins(p, lat9, ND, N, &c, path);
    if (path == 2 && !c.M[0]) return fail(MB_ERR_ARG, "the cell cannot be binned (a periodic direction is under 3 Rc wide)");
    ncell = c.M[0] ? c.M[0] * c.M[1] * c.M[2] : 1;
    if ((r = ensure(p, N, p->d.capNB ? p->d.capNB : (NM < 64 ? NM : 64), ncell))) return r;
    p->d.legs_on = 0;
    for (tries = 0; tries < 3; tries++) {
        if ((r = upload(p, N, XT, atmn, lat9, x))) return r;
        CK(cudaMemsetAsync(p->d.status, 0, sizeof(int) * 4, p->stream), "memset status");
        if ((r = mbk_wrap(&p->d, N, &c, p->stream, &p->launches))) return cuda_fail((cudaError_t)r, "wrap");
        if ((r = mbk_nlist(&p->d, N, NM, &c, p->m.rc_list, p->stream, &p->launches)))
            return cuda_fail((cudaError_t)r, "neighbour list");
        CK(cudaMemcpyAsync(p->h_status, p->d.status, sizeof(int) * 4, cudaMemcpyDeviceToHost, p->stream), "D2H status");
        CK(cudaStreamSynchronize(p->stream), "synchronize");
        if (p->h_status[0] & MB_ST_WRAP) return fail(MB_ERR_STATE, "non-finite or runaway positions");
        if (p->h_status[0] & MB_ST_NBR_OVERFLOW)
            return fail(MB_ERR_NEIGHBOURS, "an atom reached NM=%d neighbours within %.4f A; increase NM", NM, p->m.rc_list);
        if (!(p->h_status[0] & MB_ST_CAP_OVERFLOW)) break;
        if ((r = ensure(p, N, p->h_status[1] + 8, ncell))) return r;
    }
    if (tries == 3) return fail(MB_ERR_CAPACITY, "neighbour capacity could not be established");
    if (p->h_status[1] > cap) return fail(MB_ERR_CAPACITY, "an atom has %d neighbours; cap is %d", p->h_status[1], cap);
    capNB = p->d.capNB;
    hnn = (int *)malloc(sizeof(int) * N);
    hnj = (int *)malloc(sizeof(int) * (size_t)N * capNB);
    hnd = (double *)malloc(sizeof(double) * 4 * (size_t)N * capNB);
    hx = (double *)malloc(sizeof(double) * 3 * N);
    if (!hnn || !hnj || !hnd || !hx) {
        r = fail(MB_ERR_ARG, "out of host memory");
        goto out;
    }
    if (cudaMemcpy(hnn, p->d.nn, sizeof(int) * N, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(hnj, p->d.nj, sizeof(int) * (size_t)N * capNB, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(hnd, p->d.nd, sizeof(double) * 4 * (size_t)N * capNB, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(hx, p->d.X, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost) != cudaSuccess) {
        r = fail(MB_ERR_CUDA, "D2H neighbour list");
        goto out;
    }
    /* the kernels keep each entry's displacement d = S + (x_j - x_i) with
     * S = sum_q ic_q L_q; ic_q = rint(S . R_q) since L_p . R_q = delta_pq */
    for (i = 0; i < N; i++) {
        nn[i] = hnn[i];
        for (t = 0; t < hnn[i]; t++) {
            const size_t o = (size_t)i * capNB + t, w = (size_t)i * cap + t;
            const int j = hnj[o];
            double S[3];
            nj[w] = j;
            for (q = 0; q < 3; q++) S[q] = hnd[4 * o + q] - (hx[3 * j + q] - hx[3 * i + q]);
            for (q = 0; q < 3; q++)
                shift[3 * w + q] = (int)lrint(S[0] * c.R[3 * q] + S[1] * c.R[3 * q + 1] + S[2] * c.R[3 * q + 2]);
        }
    }
    if (x_wrapped) memcpy(x_wrapped, hx, sizeof(double) * 3 * N);
    r = MB_OK;
out:
    free(hnn);
    free(hnj);
    free(hnd);
    free(hx);
    return r;
}

int mb_descriptor_jvp(mb_potential *p, int N, int NM, int ND, int XT, const int *atmn, const double *lat9,
                      const double *x, const double *dx, const double *eps, double *dG) {
    mb_cell c;
    int r, tries, ncell;
    if (!p || N < 1 || NM < 1 || ND < 0 || ND > 3 || !atmn || !lat9 || !x || !dG || (!dx && !eps))
        return fail(MB_ERR_ARG, "bad arguments");
    CK(cudaSetDevice(p->device), "cudaSetDevice");
    setup_cell(p, lat9, ND, N, &c);
    ncell = c.M[0] ? c.M[0] * c.M[1] * c.M[2] : 1;
    if ((r = ensure(p, N, p->d.capNB ? p->d.capNB : (NM < 64 ? NM : 64), ncell))) return r;
    p->d.legs_on = 0;
    for (tries = 0; tries < 3; tries++) {
        if ((r = upload(p, N, XT, atmn, lat9, x))) return r;
        CK(cudaMemsetAsync(p->d.status, 0, sizeof(int) * 4, p->stream), "memset status");
        if ((r = mbk_wrap(&p->d, N, &c, p->stream, &p->launches))) return cuda_fail((cudaError_t)r, "wrap");
        if ((r = mbk_nlist(&p->d, N, NM, &c, p->m.rc_list, p->stream, &p->launches)))
            return cuda_fail((cudaError_t)r, "neighbour list");
        CK(cudaMemcpyAsync(p->h_status, p->d.status, sizeof(int) * 4, cudaMemcpyDeviceToHost, p->stream), "D2H status");
        CK(cudaStreamSynchronize(p->stream), "synchronize");
        if (p->h_status[0] & MB_ST_WRAP) return fail(MB_ERR_STATE, "non-finite or runaway positions");
        if (p->h_status[0] & MB_ST_NBR_OVERFLOW)
            return fail(MB_ERR_NEIGHBOURS, "an atom reached NM=%d neighbours within %.4f A; increase NM", NM, p->m.rc_list);
        if (!(p->h_status[0] & MB_ST_CAP_OVERFLOW)) break;
        if ((r = ensure(p, N, p->h_status[1] + 8, ncell))) return r;
    }
    if (tries == 3) return fail(MB_ERR_CAPACITY, "neighbour capacity could not be established");
    /* the displacement tangent goes to the force buffer, which no pass keeps */
    if (dx)
        CK(cudaMemcpyAsync(p->d.F, dx, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, p->stream), "H2D dx");
    else
        CK(cudaMemsetAsync(p->d.F, 0, sizeof(double) * 3 * N, p->stream), "memset dx");
    if ((r = mbk_jvp(&p->d, &p->m, N, p->d.F, eps, p->d.G, p->stream, &p->launches)))
        return cuda_fail((cudaError_t)r, "descriptor tangent kernel");
    CK(cudaMemcpyAsync(dG, p->d.G, sizeof(double) * (size_t)N * p->m.P.D, cudaMemcpyDeviceToHost, p->stream), "D2H dG");
    CK(cudaStreamSynchronize(p->stream), "synchronize");
    return MB_OK;
}

/* ------------------------------------------------------------------ */
/* relaxation (CELL_MIN, src/cmin.c)                                   */
/* ------------------------------------------------------------------ */

typedef struct {
    mb_potential *p;
    int N, NM, ND, rlxt, nfree;
    const int *atmn;
    double L[9];
    double *xf;       /* fractional coordinates */
    double *xc;       /* Cartesian scratch */
    double *F;
    double p_gpa, urep, H;
    int err;
    long ne, nf;
    /* force criterion of the last energy+gradient evaluation and its DOF */
    double maxf, maxu;
    double *last_x;
    int ndof;
} relax_ctx;

/* STR_BUF: DOF vector from the current structure (src/cmin.c:22-52) */
static void str_buf(relax_ctx *r, double *x) {
    int i, q, j = 0;
    if (r->rlxt != 7)
        for (i = 0; i < r->N; i++)
            for (q = 0; q < 3; q++) x[j++] = r->xf[3 * i + q];
    if (r->rlxt == 2) return;
    if (r->rlxt > 7) { x[j++] = r->L[8]; return; }
    x[j++] = r->L[0]; x[j++] = r->L[4]; x[j++] = r->L[8];
    x[j++] = r->L[1]; x[j++] = r->L[5]; x[j++] = r->L[6];
    x[j++] = r->L[3]; x[j++] = r->L[7]; x[j++] = r->L[2];
}

/* BUF_STR: structure from the DOF vector (src/cmin.c:54-88) */
static void buf_str(relax_ctx *r, const double *x) {
    int i, q, j = 0;
    if (r->rlxt != 7)
        for (i = 0; i < r->N; i++)
            for (q = 0; q < 3; q++) r->xf[3 * i + q] = x[j++];
    if (r->rlxt == 2) return;
    if (r->rlxt > 7) { r->L[8] = x[j++]; return; }
    r->L[0] = x[j++]; r->L[4] = x[j++]; r->L[8] = x[j++];
    r->L[1] = x[j++]; r->L[5] = x[j++]; r->L[6] = x[j++];
    r->L[3] = x[j++]; r->L[7] = x[j++]; r->L[2] = x[j++];
}

/* Relative(): Cartesian -> fractional with the reference's sums (src/cell.c:445-465) */
static void cart_to_frac(int N, const double *x, const double *L, double *xf) {
    double R[9];
    int i, q, j;
    reciprocal(L, R);
    for (i = 0; i < N; i++)
        for (q = 0; q < 3; q++) {
            double s = 0.0;
            for (j = 0; j < 3; j++) s += x[3 * i + j] * R[3 * q + j];
            xf[3 * i + q] = s;
        }
}

/* evaluate at DOF x; afterwards x holds the wrapped structure (src/cmin.c:90-166) */
static double relax_eval(relax_ctx *r, double *x, double *g) {
    int rc, i, q, k, j = 0;
    buf_str(r, x);
    frac_to_cart(r->N, r->xf, r->L, r->xc);
    if (r->err) return NAN;
    if (!g) {
        rc = mb_energy(r->p, r->N, r->NM, r->ND, 1, r->atmn, r->L, r->xc, r->p_gpa, r->urep, &r->H, NULL, NULL);
        r->ne++;
        if (!rc && r->p->res_staged)
            memcpy(r->xc, r->p->h_res + 3 * r->N, sizeof(double) * 3 * r->N);
        else if (!rc && cudaMemcpy(r->xc, r->p->d.X, sizeof(double) * 3 * r->N, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = fail(MB_ERR_CUDA, "D2H positions");
        if (rc) { r->err = rc; return NAN; }
    } else {
        double U[6], R[9], V = cell_volume(r->L);
        reciprocal(r->L, R);
        rc = mb_efs(r->p, r->N, r->NM, r->ND, 1, r->atmn, r->L, r->xc, r->p_gpa, r->urep, &r->H, NULL, r->F, U, NULL,
                    r->xc);
        r->nf++;
        if (rc) { r->err = rc; return NAN; }
        if (r->rlxt != 7)
            for (i = 0; i < r->N; i++)
                for (q = 0; q < 3; q++) {
                    double d = 0.0;
                    for (k = 0; k < 3; k++) d = d - r->F[3 * i + k] * r->L[3 * q + k];
                    g[j++] = d;
                }
        if (r->rlxt != 2) {
            double pv = r->p_gpa / MB_EV2GPA * V;
            for (q = 0; q < 3; q++) U[q] -= pv;
            if (r->rlxt > 7)
                g[j++] = -(U[2] * R[8]);
            else {
                g[j++] = -(U[0] * R[0] + U[3] * R[1] + U[5] * R[2]);
                g[j++] = -(U[3] * R[3] + U[1] * R[4] + U[4] * R[5]);
                g[j++] = -(U[5] * R[6] + U[4] * R[7] + U[2] * R[8]);
                g[j++] = -(U[3] * R[0] + U[1] * R[1] + U[4] * R[2]);
                g[j++] = -(U[5] * R[3] + U[4] * R[4] + U[2] * R[5]);
                g[j++] = -(U[0] * R[6] + U[3] * R[7] + U[5] * R[8]);
                g[j++] = -(U[0] * R[3] + U[3] * R[4] + U[5] * R[5]);
                g[j++] = -(U[3] * R[6] + U[1] * R[7] + U[4] * R[8]);
                g[j++] = -(U[5] * R[0] + U[4] * R[1] + U[2] * R[2]);
            }
        }
        for (i = 0; i < j; i++)
            if (fabs(g[i]) < 1e-10) g[i] = 0.0;
        /* force criterion at this point: max |F| and max |U - pV| / N */
        {
            double mf = 0.0, mu = 0.0, pv = r->p_gpa / MB_EV2GPA * V;
            for (i = 0; i < 3 * r->N; i++)
                if (fabs(r->F[i]) > mf) mf = fabs(r->F[i]);
            for (q = 0; q < 6; q++) {
                double u = (r->rlxt == 2) ? 0.0 : fabs(U[q]) / r->N;
                if (u > mu) mu = u;
            }
            (void)pv;
            r->maxf = mf;
            r->maxu = mu;
        }
    }
    /* STR_BUF after the wrap performed by the list build */
    cart_to_frac(r->N, r->xc, r->L, r->xf);
    str_buf(r, x);
    if (g && r->last_x) memcpy(r->last_x, x, sizeof(double) * r->ndof);
    return r->H;
}

static double relax_f(void *ctx, double *x) { return relax_eval((relax_ctx *)ctx, x, NULL); }
static double relax_fg(void *ctx, double *x, double *g) { return relax_eval((relax_ctx *)ctx, x, g); }

/* Relaxation with the force criterion (see mb_relax_fmax): the same DOF
 * mapping and BFGS, line-search tolerance 0.1. */
int mb_relax_fmax(mb_potential *p, int N, int NM, int ND, const int *atmn, double *lat9, double *x, double p_gpa,
                  double urep, int rlxt, int mitr, double fmax, double *H, long *counts, int *converged) {
    relax_ctx r;
    mb_bfgs b;
    double *dof, *gtmp;
    int n, iter = 0, rc = MB_OK, st, conv = 0;
    if (!p || N < 1 || !atmn || !lat9 || !x || !(fmax > 0)) return fail(MB_ERR_ARG, "bad arguments");
    if (!(rlxt == 2 || rlxt == 3)) return fail(MB_ERR_ARG, "RLXT %d not supported here (2, 3)", rlxt);
    memset(&r, 0, sizeof(r));
    r.p = p; r.N = N; r.NM = NM; r.ND = ND; r.rlxt = rlxt; r.atmn = atmn; r.p_gpa = p_gpa; r.urep = urep;
    memcpy(r.L, lat9, sizeof(double) * 9);
    n = 3 * N + (rlxt == 3 ? 9 : 0);
    r.ndof = n;
    r.xf = (double *)malloc(sizeof(double) * 3 * N);
    r.xc = (double *)malloc(sizeof(double) * 3 * N);
    r.F = (double *)malloc(sizeof(double) * 3 * N);
    r.last_x = (double *)malloc(sizeof(double) * n);
    dof = (double *)malloc(sizeof(double) * n);
    gtmp = (double *)malloc(sizeof(double) * n);
    memcpy(r.xc, x, sizeof(double) * 3 * N);
    cart_to_frac(N, r.xc, r.L, r.xf);
    str_buf(&r, dof);
    if (mb_bfgs_init(&b, n, dof, 0.01, 0.1, relax_f, relax_fg, &r)) { rc = fail(MB_ERR_ARG, "out of memory"); goto done; }
    if (r.err) { rc = r.err; mb_bfgs_free(&b); goto done; }
    conv = r.maxf < fmax && r.maxu < fmax;
    while (!conv && iter < mitr) {
        iter++;
        st = mb_bfgs_iterate(&b);
        if (r.err) { rc = r.err; break; }
        if (st != MB_BFGS_OK) break;
        if (memcmp(r.last_x, b.x, sizeof(double) * n) != 0) {
            /* accepted point is not the last evaluated one: refresh the criterion there */
            memcpy(dof, b.x, sizeof(double) * n);
            relax_fg(&r, dof, gtmp);
            if (r.err) { rc = r.err; break; }
        }
        conv = r.maxf < fmax && r.maxu < fmax;
    }
    if (!rc) {
        buf_str(&r, b.x);
        frac_to_cart(N, r.xf, r.L, x);
        memcpy(lat9, r.L, sizeof(double) * 9);
        if (H) *H = b.f;
        if (counts) { counts[0] = r.ne; counts[1] = r.nf; counts[2] = iter; }
        if (converged) *converged = conv;
    }
    mb_bfgs_free(&b);
done:
    free(r.xf); free(r.xc); free(r.F); free(r.last_x); free(dof); free(gtmp);
    return rc;
}

int mb_relax(mb_potential *p, int N, int NM, int ND, const int *atmn, double *lat9, double *x, double p_gpa,
             double urep, int rlxt, int mitr, double etol, double *H, long *counts) {
    relax_ctx r;
    mb_bfgs b;
    double *dof, E;
    int n, iter = 0, rc = MB_OK, st;
    if (!p || N < 1 || !atmn || !lat9 || !x) return fail(MB_ERR_ARG, "bad arguments");
    if (!(rlxt == 2 || rlxt == 3 || rlxt == 7 || rlxt == 8)) return fail(MB_ERR_ARG, "RLXT %d not supported (2, 3, 7, 8)", rlxt);
    memset(&r, 0, sizeof(r));
    r.p = p; r.N = N; r.NM = NM; r.ND = ND; r.rlxt = rlxt; r.atmn = atmn; r.p_gpa = p_gpa; r.urep = urep;
    memcpy(r.L, lat9, sizeof(double) * 9);
    r.xf = (double *)malloc(sizeof(double) * 3 * N);
    r.xc = (double *)malloc(sizeof(double) * 3 * N);
    r.F = (double *)malloc(sizeof(double) * 3 * N);
    n = (rlxt != 7 ? 3 * N : 0) + (rlxt == 3 || rlxt == 7 ? 9 : 0) + (rlxt == 8 ? 1 : 0);
    dof = (double *)malloc(sizeof(double) * n);
    /* CELL_RELX evaluates E+F+S first, which also wraps the positions (src/cmod.c:922) */
    rc = mb_efs(p, N, NM, ND, 1, atmn, r.L, x, p_gpa, urep, &r.H, NULL, r.F, NULL, NULL, r.xc);
    if (rc) goto done;
    cart_to_frac(N, r.xc, r.L, r.xf);
    str_buf(&r, dof);
    /* CELL_MIN: O = cfunc(p); minimiser set with step 0.01 and tolerance 0.001 (src/cmin.c:237-245) */
    relax_f(&r, dof);
    if (r.err) { rc = r.err; goto done; }
    if (mb_bfgs_init(&b, n, dof, 0.01, 0.001, relax_f, relax_fg, &r)) { rc = fail(MB_ERR_ARG, "out of memory"); goto done; }
    if (r.err) { rc = r.err; mb_bfgs_free(&b); goto done; }
    E = r.H;
    do {
        iter++;
        st = mb_bfgs_iterate(&b);
        if (r.err) { rc = r.err; break; }
        if (st != MB_BFGS_OK) break; /* no further progress possible from this state */
        /* gsl_multimin_test_size(|H - H_prev|, ETOL) */
        if (fabs(r.H - E) < etol) { E = r.H; break; }
        E = r.H;
    } while (iter < mitr);
    if (!rc) {
        /* final structure = minimiser state (src/cmin.c:284-286) */
        buf_str(&r, b.x);
        frac_to_cart(N, r.xf, r.L, x);
        memcpy(lat9, r.L, sizeof(double) * 9);
        if (H) *H = b.f;
        if (counts) { counts[0] = r.ne; counts[1] = r.nf; counts[2] = iter; }
    }
    mb_bfgs_free(&b);
done:
    free(r.xf); free(r.xc); free(r.F); free(dof);
    return rc;
}

/* ------------------------------------------------------------------ */
/* NVT molecular dynamics                                              */
/* ------------------------------------------------------------------ */

/* Move the times of the recorded step and kernel events into the
 * accumulators and free the pool slots (the stream must be idle). */
static int harvest_events(mb_potential *p) {
    int k;
    for (k = 0; k < p->d.st_n; k++) {
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, ((cudaEvent_t *)p->d.st_pool)[2 * k], ((cudaEvent_t *)p->d.st_pool)[2 * k + 1]),
           "cudaEventElapsedTime");
        p->st_acc_ms += ms;
        p->st_acc_n++;
    }
    for (k = 0; k < p->d.ev_n; k++) {
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, ((cudaEvent_t *)p->d.ev_pool)[2 * k], ((cudaEvent_t *)p->d.ev_pool)[2 * k + 1]),
           "cudaEventElapsedTime");
        p->ev_acc_ms += ms;
        p->ev_acc_n++;
    }
    p->d.st_n = 0;
    p->d.ev_n = 0;
    return MB_OK;
}

/* One MD step of Dynamics' NVT branch: CELL_FRC (wrap + list + descriptor
 * pass + finalize), thermostat and integrator, then JAR.  With step
 * profiling on, the L2 is overwritten before the step, outside its events. */
static int md_step(mb_potential *p, int N, int NM, const mb_cell *c, double urep, double dt, double tau, double T,
                   int tag) {
    cudaEvent_t t1 = 0;
    int r;
    if (p->d.st_on && p->d.flush)
        CK(cudaMemsetAsync(p->d.flush, tag & 0xff, p->d.flush_bytes, p->stream), "flush");
    if (p->d.st_on && p->d.st_n < p->d.st_cap) {
        mbk_record(((cudaEvent_t *)p->d.st_pool)[2 * p->d.st_n], p->stream);
        t1 = ((cudaEvent_t *)p->d.st_pool)[2 * p->d.st_n + 1];
        p->d.st_n++;
    }
    if ((r = mbk_wrap(&p->d, N, c, p->stream, &p->launches))) return cuda_fail((cudaError_t)r, "wrap");
    if ((r = mbk_nlist(&p->d, N, NM, c, p->m.rc_list, p->stream, &p->launches)))
        return cuda_fail((cudaError_t)r, "neighbour list");
    if ((r = mbk_descriptor_pass(&p->d, &p->m, N, MB_MODE_EFS, urep, 0, 0, p->stream, &p->launches)))
        return cuda_fail((cudaError_t)r, "descriptor kernel");
    if ((r = mbk_finalize(&p->d, N, MB_MODE_EFS, 0.0, p->stream, &p->launches)))
        return cuda_fail((cudaError_t)r, "finalize");
    if ((r = mbk_nvt_update(&p->d, &p->m, N, dt, tau, T / MB_KB_INV, c, p->stream, &p->launches)))
        return cuda_fail((cudaError_t)r, "integrator");
    if (t1) mbk_record(t1, p->stream);
    return MB_OK;
}

/* Queue `chunk` MD steps from `step` on.  They run as one CUDA graph,
 * captured on first use and replayed while nothing it was captured for has
 * changed; a chunk whose kernel shape is not tuned yet (tuning times launches
 * and synchronises) runs as plain launches.  *graphed tells which. */
static int md_chunk(mb_potential *p, int N, int NM, const mb_cell *c, double urep, double dt, double tau, double T,
                    int step, int chunk, int *graphed) {
    int r, s;
    *graphed = 0;
    p->d.legs_on = mbk_legs_usable(&p->d, &p->m, N, c);
    CK(cudaMemsetAsync(p->d.status, 0, sizeof(int) * 4, p->stream), "memset status");
    if ((r = mbk_set_out(&p->d, 10, (double)step, p->stream))) return cuda_fail((cudaError_t)r, "set step");
    if (p->use_graphs && mbk_shape_ready(&p->d, N, MB_MODE_EFS)) {
        md_key k;
        memset(&k, 0, sizeof(k));
        k.gen = p->gen;
        k.N = N;
        k.NM = NM;
        k.chunk = chunk;
        k.st_on = p->d.st_on;
        k.ev_on = p->d.ev_on;
        k.urep = urep;
        k.dt = dt;
        k.tau = tau;
        k.T = T;
        k.c = *c;
        k.flush = p->d.flush;
        k.flush_bytes = p->d.flush_bytes;
        k.trace = p->d.trace;
        k.st_pool = p->d.st_pool;
        k.ev_pool = p->d.ev_pool;
        k.legs = p->d.legs_on;
        if (!p->md_exec || memcmp(&k, &p->md_k, sizeof(k))) {
            cudaGraph_t g = NULL;
            cudaError_t e;
            const long l0 = p->launches;
            if (p->md_exec) {
                cudaGraphExecDestroy(p->md_exec);
                p->md_exec = NULL;
            }
            /* the captured events take the first pool slots */
            CK(cudaStreamSynchronize(p->stream), "synchronize");
            if ((r = harvest_events(p))) return r;
            CK(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            for (s = 0; s < chunk; s++)
                if ((r = md_step(p, N, NM, c, urep, dt, tau, T, s))) break;
            e = cudaStreamEndCapture(p->stream, &g);
            if (r) {
                if (g) cudaGraphDestroy(g);
                return r;
            }
            if (e != cudaSuccess) return cuda_fail(e, "end capture");
            e = cudaGraphInstantiate(&p->md_exec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                p->md_exec = NULL;
                return cuda_fail(e, "graph instantiate");
            }
            p->md_k = k;
            p->md_launches = p->launches - l0;
            p->launches = l0;
            p->md_st_events = p->d.st_n;
            p->md_ev_events = p->d.ev_n;
            p->d.st_n = 0;
            p->d.ev_n = 0;
        }
        CK(cudaGraphLaunch(p->md_exec, p->stream), "graph launch");
        p->launches += p->md_launches;
        *graphed = 1;
        return MB_OK;
    }
    for (s = 0; s < chunk; s++)
        if ((r = md_step(p, N, NM, c, urep, dt, tau, T, step + s))) return r;
    return MB_OK;
}

int mb_md_nvt(mb_potential *p, int N, int NM, int ND, const int *atmn, const double *lat9, double *x, double *v,
              double T, double dt, double tau, int nsteps, double urep, double *xi, double *Hs, double *Ks) {
    mb_cell c;
    int r, step, chunk;
    double xi0 = xi ? *xi : 0.0, *X0, *V0;
    if (!p || N < 1 || !atmn || !lat9 || !x || !v || nsteps < 0 || !(T > 0) || !(tau > 0))
        return fail(MB_ERR_ARG, "bad arguments");
    CK(cudaSetDevice(p->device), "cudaSetDevice");
    setup_cell(p, lat9, ND, N, &c);
    if ((r = ensure(p, N, p->d.capNB ? p->d.capNB : (NM < 64 ? NM : 64), c.M[0] ? c.M[0] * c.M[1] * c.M[2] : 1)))
        return r;
    if ((r = upload(p, N, 1, atmn, lat9, x))) return r;
    CK(cudaMemcpyAsync(p->d.V, v, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, p->stream), "H2D velocities");
    if (p->d.capTrace < nsteps) {
        cudaFree(p->d.trace);
        CK(cudaMalloc((void **)&p->d.trace, sizeof(double) * 2 * (nsteps > 0 ? nsteps : 1)), "alloc trace");
        p->d.capTrace = nsteps;
    }
    /* establish the neighbour capacity once (wraps the positions, as JAR before the loop) */
    r = run_pass(p, N, NM, ND, lat9, MB_MODE_EFS, urep, 0.0);
    if (r == MB_RETRY) {
        if ((r = upload(p, N, 1, atmn, lat9, x))) return r;
        r = run_pass(p, N, NM, ND, lat9, MB_MODE_EFS, urep, 0.0);
    }
    if (r) return r == MB_RETRY ? fail(MB_ERR_CAPACITY, "neighbour capacity could not be established") : r;
    if ((r = mbk_set_out(&p->d, 9, xi0, p->stream))) return cuda_fail((cudaError_t)r, "set xi");
    /* checkpoints for re-running a chunk whose neighbour counts outgrew the capacity */
    CK(cudaMalloc((void **)&X0, sizeof(double) * 3 * N), "alloc checkpoint");
    CK(cudaMalloc((void **)&V0, sizeof(double) * 3 * N), "alloc checkpoint");
    for (step = 0; step < nsteps; step += chunk) {
        int attempt, graphed = 0;
        double xis;
        chunk = nsteps - step < 10 ? nsteps - step : 10;
        CK(cudaMemcpyAsync(X0, p->d.X, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, p->stream), "checkpoint");
        CK(cudaMemcpyAsync(V0, p->d.V, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, p->stream), "checkpoint");
        CK(cudaMemcpyAsync(p->h_out, p->d.out, sizeof(double) * 16, cudaMemcpyDeviceToHost, p->stream), "D2H out");
        CK(cudaStreamSynchronize(p->stream), "synchronize");
        xis = p->h_out[9];
        for (attempt = 0; attempt < 3; attempt++) {
            const int st0 = p->d.st_n, ev0 = p->d.ev_n;
            if ((r = md_chunk(p, N, NM, &c, urep, dt, tau, T, step, chunk, &graphed))) goto out;
            CK(cudaMemcpyAsync(p->h_status, p->d.status, sizeof(int) * 4, cudaMemcpyDeviceToHost, p->stream), "D2H status");
            CK(cudaStreamSynchronize(p->stream), "synchronize");
            if (p->h_status[0] & MB_ST_WRAP) { r = fail(MB_ERR_STATE, "non-finite positions in MD"); goto out; }
            if (p->h_status[0] & MB_ST_NBR_OVERFLOW) {
                r = fail(MB_ERR_NEIGHBOURS, "an atom reached NM=%d neighbours during MD", NM);
                goto out;
            }
            if (!(p->h_status[0] & MB_ST_CAP_OVERFLOW)) {
                if (graphed) {
                    /* the replay re-recorded the graph's events: move their times out */
                    p->d.st_n = p->md_st_events;
                    p->d.ev_n = p->md_ev_events;
                    if ((r = harvest_events(p))) goto out;
                }
                break;
            }
            /* grow and replay the chunk from its checkpoint (its timings are dropped) */
            p->d.st_n = graphed ? 0 : st0;
            p->d.ev_n = graphed ? 0 : ev0;
            if ((r = ensure(p, N, p->h_status[1] + 8, c.M[0] ? c.M[0] * c.M[1] * c.M[2] : 1))) goto out;
            CK(cudaMemcpyAsync(p->d.X, X0, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, p->stream), "restore");
            CK(cudaMemcpyAsync(p->d.V, V0, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, p->stream), "restore");
            if ((r = mbk_set_out(&p->d, 9, xis, p->stream))) { r = cuda_fail((cudaError_t)r, "set xi"); goto out; }
        }
        if (attempt == 3) { r = fail(MB_ERR_CAPACITY, "neighbour capacity could not be established"); goto out; }
    }
    CK(cudaMemcpyAsync(x, p->d.X, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, p->stream), "D2H X");
    CK(cudaMemcpyAsync(v, p->d.V, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, p->stream), "D2H V");
    CK(cudaMemcpyAsync(p->h_out, p->d.out, sizeof(double) * 16, cudaMemcpyDeviceToHost, p->stream), "D2H out");
    if (nsteps > 0 && (Hs || Ks)) {
        double *tr = (double *)malloc(sizeof(double) * 2 * nsteps);
        int k;
        CK(cudaMemcpyAsync(tr, p->d.trace, sizeof(double) * 2 * nsteps, cudaMemcpyDeviceToHost, p->stream), "D2H trace");
        CK(cudaStreamSynchronize(p->stream), "synchronize");
        for (k = 0; k < nsteps; k++) {
            if (Hs) Hs[k] = tr[2 * k];
            if (Ks) Ks[k] = tr[2 * k + 1];
        }
        free(tr);
    }
    CK(cudaStreamSynchronize(p->stream), "synchronize");
    if (xi) *xi = p->h_out[9];
    r = MB_OK;
out:
    cudaFree(X0);
    cudaFree(V0);
    return r;
}

/* ------------------------------------------------------------------ */
/* Maxwell velocities with the reference's random streams              */
/* ------------------------------------------------------------------ */

/* Lehmer generator x <- 48271 x mod (2^31-1) with 256 streams spaced by the
 * jump multiplier 22925 (Park & Miller 1988; Park & Geyer's rngs
 * library), evaluated with Schrage's decomposition to stay in 32-bit range.
 * Only stream 0 is drawn, as the reference does. */
typedef struct {
    long seed[256];
} mb_rng;

static long lehmer(long x, long a) {
    const long m = 2147483647, q = m / a, r = m % a;
    long t = a * (x % q) - r * (x / q);
    return t > 0 ? t : t + m;
}

static void rng_plant(mb_rng *g, long x) {
    int j;
    if (x > 0) x %= 2147483647;
    g->seed[0] = x;
    for (j = 1; j < 256; j++) g->seed[j] = lehmer(g->seed[j - 1], 22925);
}

static double rng_next(mb_rng *g) {
    g->seed[0] = lehmer(g->seed[0], 48271);
    return (double)g->seed[0] / 2147483647.0;
}

int mb_maxwell(int N, const double *amu, double T, long seed, double *v) {
    mb_rng g;
    double vv, Vc[3] = {0, 0, 0}, s = 0.0;
    int i, q;
    if (N < 1 || !amu || !v || !(T > 0) || seed <= 0) return fail(MB_ERR_ARG, "bad arguments");
    rng_plant(&g, seed);
    /* src/cmod.c:249-278 with every atom free; T in K, kT in eV */
    vv = sqrt(3.0 * (T / MB_KB_INV));
    for (i = 0; i < N; i++) {
        double m = amu[i] * 103.6427;
        double f = rng_next(&g) * 2.0 * MB_PI;
        double Q = rng_next(&g) * MB_PI;
        v[3 * i] = vv * sin(Q) * cos(f) / sqrt(m);
        v[3 * i + 1] = vv * sin(Q) * sin(f) / sqrt(m);
        v[3 * i + 2] = vv * cos(Q) / sqrt(m);
        for (q = 0; q < 3; q++) Vc[q] += v[3 * i + q];
    }
    for (i = 0; i < N; i++)
        for (q = 0; q < 3; q++) v[3 * i + q] -= Vc[q] / (double)N;
    for (i = 0; i < N; i++)
        for (q = 0; q < 3; q++) s += v[3 * i + q] * v[3 * i + q] * (amu[i] * 103.6427);
    s = vv / sqrt(s / (double)N);
    for (i = 0; i < 3 * N; i++) v[i] *= s;
    return MB_OK;
}
