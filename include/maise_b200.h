/*
 * maise_b200.h -- C-ABI of the B200 implementation of MAISE's neural-network
 * interatomic potential: Behler-Parrinello G2/G4 descriptors, per-species MLP
 * energy with back-propagation to forces and virial, and the relaxation and
 * NVT molecular-dynamics drivers that consume them.
 *
 * All entry points take plain pointers and sizes.  Host arrays are row-major:
 *   x[3N]     positions (Cartesian unless stated; Angstrom)
 *   lat9[9]   lattice vectors as rows, lat9[3*i+q] = component q of vector i
 *   atmn[N]   species index of each atom in model order (0..nspc-1)
 *   frc[3N]   forces (eV/Angstrom)
 *   str[6]    virial U (eV, not divided by volume), order xx,yy,zz,xy,yz,zx
 * Units and conventions are those of the reference (src/cmod.c:1136-1163).
 *
 * Every function returns MB_OK (0) or an MB_ERR_* code; mb_last_error()
 * returns the message of the last failure in the calling thread.  Handles
 * are not thread-safe: use one per host thread.
 */
#ifndef MAISE_B200_H
#define MAISE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
    MB_OK = 0,
    MB_ERR_ARG = 1,        /* invalid argument */
    MB_ERR_MODEL = 2,      /* model/basis file missing or malformed */
    MB_ERR_NEIGHBOURS = 3, /* an atom reached NM neighbours (src/cell.c:134-142) */
    MB_ERR_CUDA = 4,       /* CUDA runtime error */
    MB_ERR_CAPACITY = 5,   /* structure larger than the reserved capacity */
    MB_ERR_NOGPU = 6,      /* no usable sm_100 device */
    MB_ERR_STATE = 7       /* invalid positions (non-finite, or wrap did not terminate) */
};

typedef struct mb_potential mb_potential;

/* Message of the last error in this thread ("" if none). */
const char *mb_last_error(void);

/* Load a MAISE 'model' file (header, input ranges, weights and the appended
 * basis) onto CUDA device `device`.
 * Replaces the first-call initialisation of CALL_MAISE: READ_MODEL
 * (src/util.c:1233-1335), Build_ANN/READ_ANN (src/nutl.c:305-357, 502-633)
 * and Build_PRS (src/nprs.c:75-257). */
int mb_open(const char *model_path, int device, mb_potential **out);
int mb_close(mb_potential *pot);

/* Model facts: number of species, their atomic numbers (spcz[nspc]),
 * descriptor length D and the neighbour-list cutoff (Angstrom). */
int mb_model_info(const mb_potential *pot, int *nspc, int *spcz, int *D, double *rc);

/* Reserve device storage for structures of up to max_atoms atoms and
 * max_neighbours neighbours per atom.  Optional: calls grow it on demand.
 * Replaces the sizing done by Build_Cell/Build_LNK (src/cell.c:6-78,
 * src/nutl.c:359-392), without their N x NM x NM angle tables. */
int mb_reserve(mb_potential *pot, int max_atoms, int max_neighbours);

/* Energy, forces and virial of one structure (CELL_FRC, src/cmod.c:153-191).
 *   NM     neighbour cap: an atom with NM neighbours is an error, as in LIST
 *   ND     number of periodic lattice directions (0 cluster, 3 crystal)
 *   XT     0: x is fractional, 1: Cartesian (src/cmod.c:1108-1117)
 *   p_gpa  external pressure; H = E + p V when ND == 3
 *   urep   short-range repulsion strength U (eV); 0 disables (src/cmod.c:61-126)
 * Outputs (any may be NULL): H, E, frc[3N], str[6], ea[N] (MLP per-atom
 * energies), x_wrapped[3N] (positions after the wrap into the cell that
 * LIST performs, src/cell.c:90-91).  |F|,|U| < 1e-8 are zeroed as in the
 * reference. */
int mb_efs(mb_potential *pot, int N, int NM, int ND, int XT, const int *atmn, const double *lat9, const double *x,
           double p_gpa, double urep, double *H, double *E, double *frc, double *str, double *ea, double *x_wrapped);

/* Energy only (CELL_ENE, src/cmod.c:128-151): descriptors + MLP forward. */
int mb_energy(mb_potential *pot, int N, int NM, int ND, int XT, const int *atmn, const double *lat9, const double *x,
              double p_gpa, double urep, double *H, double *E, double *ea);

/* Descriptor vectors G[N*D] in the reference's species-resolved layout
 * (the energy part of PRS_BP, src/nprs.c:445-566; L->Cn). */
int mb_descriptors(mb_potential *pot, int N, int NM, int ND, int XT, const int *atmn, const double *lat9,
                   const double *x, double *G);

/* Vector-Jacobian product of the descriptor map with caller weights
 * g[N*D]:  frc[i] = -sum_j sum_m g[j][m] dG_j,m/dx_i  and
 * str = -sum_i sum_m g[i][m] dG_i,m/d(strain), i.e. the contraction
 * FRC_ANN performs on Fn/Sn (src/nmlp.c:433-479) with dE/dG replaced by g.
 * No noise zeroing is applied. */
int mb_descriptor_vjp(mb_potential *pot, int N, int NM, int ND, int XT, const int *atmn, const double *lat9,
                      const double *x, const double *g, double *frc, double *str);

/* Tangent of the descriptor map: dG[N*D] = sum_i (dG/dx_i) . dx_i plus the
 * response to the homogeneous deformation d -> d + eps d of every neighbour
 * displacement (eps[9] row-major; either dx or eps may be NULL), with the
 * derivative parameters of PRS_BP's derivative part (src/nprs.c:567-770).
 * A unit dx on atom i and axis q is column q of the reference's blocks
 * Fn[i][.] (dG_j/dx_i for every j); eps = e_a e_b^T is the (a, b) column
 * of Sn (dG/dstrain, in the virial's convention d_a -> d_a + d_b).  The
 * adjoint of mb_descriptor_vjp: sum g . dG = -(frc . dx). */
int mb_descriptor_jvp(mb_potential *pot, int N, int NM, int ND, int XT, const int *atmn, const double *lat9,
                      const double *x, const double *dx, const double *eps, double *dG);

/* One structure's descriptor file <dir>/e%06d in the layout of LNK_OUT
 * (src/nprs.c:380-442), as PARS_DAT writes it for training
 * (src/nprs.c:983-1366): EFS 0 energies only, 1 with derivative blocks of
 * the marked atoms (marked[N] != 0; their reference forces frc_ref[3N], may
 * be NULL), 2 with strain blocks of every atom and the reference stresses
 * str_ref[6] (may be NULL), 3 both.  E, p, DE: the structure's reference
 * energy, pressure and energy spread for the header; data_path the source
 * directory recorded in the file.  Neighbour blocks are listed in
 * ascending atom index; an atom that is its own periodic neighbour has its
 * whole dG_i/dx_i in the self block (the reference splits off the part
 * through i's images into a block listed under i). */
int mb_parse_efile(mb_potential *pot, const char *dir, int index, int EFS, int N, int NM, int ND, int XT,
                   const int *atmn, const double *lat9, const double *x, double E, double p, double DE,
                   const int *marked, const double *frc_ref, const double *str_ref, const char *data_path);

/* The neighbour list the E/F/S passes build (LIST, src/cell.c:82-185): for
 * every atom i each (atom j, lattice image) with |x_j + S - x_i|^2 < Rc^2
 * (strict), S = sum_q shift_q L_q, excluding i's own zero image, after the
 * wrap into the cell that LIST performs.  The set is the reference's; the
 * order within an atom's list is not (LIST swaps the nearest into slot 0).
 *   path   0 as the passes choose, 1 the all-pairs search, 2 the cell list
 *          (MB_ERR_ARG if a periodic direction is under 3 Rc wide)
 *   cap    row length of nj and shift
 * Outputs: nn[N] counts, nj[N*cap] neighbour atoms, shift[N*cap*3] integer
 * images, x_wrapped[3N] (may be NULL).  MB_ERR_CAPACITY if an atom has more
 * than cap neighbours; MB_ERR_NEIGHBOURS if one reaches NM. */
int mb_neighbours(mb_potential *pot, int N, int NM, int ND, int XT, const int *atmn, const double *lat9,
                  const double *x, int path, int cap, int *nn, int *nj, int *shift, double *x_wrapped);

/* Cell relaxation (CELL_RELX/CELL_MIN, src/cmod.c:901-977,
 * src/cmin.c:22-301).  Degrees of freedom as STR_BUF: fractional atom
 * coordinates (rlxt 2), plus the 9 lattice components (rlxt 3), or the
 * lattice only (rlxt 7).  BFGS with Fletcher's line search (step 0.01,
 * tolerance 0.001); stops when |H - H_prev| < etol or after mitr
 * iterations.  lat9 and x (Cartesian) are updated in place.
 * counts (may be NULL) receives {energy calls, force calls, iterations}. */
int mb_relax(mb_potential *pot, int N, int NM, int ND, const int *atmn, double *lat9, double *x, double p_gpa,
             double urep, int rlxt, int mitr, double etol, double *H, long *counts);

/* mb_relax with the force criterion of mb_relax_batch instead of the
 * enthalpy change: stops when max |F| < fmax and max |U - pV| / N < fmax,
 * or after mitr iterations.  Returns MB_OK; *converged tells which. */
int mb_relax_fmax(mb_potential *pot, int N, int NM, int ND, const int *atmn, double *lat9, double *x, double p_gpa,
                  double urep, int rlxt, int mitr, double fmax, double *H, long *counts, int *converged);

/* Relaxation of a population of independent structures in one persistent
 * launch: the batched counterpart of the evolutionary search's serial
 * relaxation loop (RELX_INT, src/emod.c:521-548, each member through
 * CELL_RELX).  Structure s has nat[s] <= 64 atoms; its atoms are rows
 * off[s] .. off[s]+nat[s]-1 of atmn and x (off = exclusive prefix sum of
 * nat); lat[9*s] is its lattice.  Every structure is relaxed on the device
 * by BFGS with Fletcher's line search over the DOF vector of rlxt (2 or 3),
 * FP64 state, with descriptors and MLP in FP32 and FP64 energy and virial
 * reductions.  A structure stops when max |F| < fmax (eV/A) and
 * max |U_ab - pV delta_ab| / N < fmax (eV), or after mitr iterations.
 * x (Cartesian) and lat are updated in place; H[s] gets the enthalpy,
 * iters[s] the iterations and status[s] 0 (converged), 1 (iteration limit),
 * 2 (too many neighbours), 3 (no descent possible). */
int mb_relax_batch(mb_potential *pot, int S, const int *nat, const int *atmn, double *lat, double *x, double p_gpa,
                   double urep, int rlxt, int mitr, double fmax, double *H, int *iters, int *status);

/* Energy, forces and virial of every structure of a population, computed
 * by the evaluation of mb_relax_batch (FP32 descriptors and MLP, FP64
 * energy and virial reductions) without relaxing: the batched counterpart
 * of CELL_FRC (src/cmod.c:153-191) over RELX_INT's members.  Layout and
 * limits as mb_relax_batch (nat[s] <= 64, at most 96 neighbours per atom);
 * x Cartesian.  Outputs: H[S] enthalpies (E + pV), frc[3 * sum nat] forces,
 * str[6S] virials U (may be NULL).  No noise zeroing.  Stated error of the
 * FP32 evaluation against mb_efs: at most 1e-5 eV/atom in energy and
 * 1e-4 eV/A in force. */
int mb_efs_batch(mb_potential *pot, int S, const int *nat, const int *atmn, const double *lat, const double *x,
                 double p_gpa, double urep, double *H, double *frc, double *str);

/* ---- evolutionary search hand-off (src/emod.c) ---- */

/* The batched drop-in for RELX_INT (src/emod.c:521-548): relax S offspring
 * in one mb_relax_batch launch and write member p0 + s of generation gen to
 * <evos_dir>/G%03d/M%03d/ as the reference leaves it for RELX_TR
 * (src/emod.c:710-718): POSCAR.0 (the structure before relaxing),
 * CONTCAR.0 (after; SAVE_CELL's layout, src/util.c:991-1060), OSZICAR.0
 * (the enthalpy line Read_OSZI reads, src/util.c:1130-1147) and OUTCAR.0
 * (CELL_OUT's final block with forces and stress, src/cmod.c:617-685).
 * Arguments and in-place updates as mb_relax_batch; atoms of each structure
 * grouped by species.  Species symbols are the model's. */
int mb_evos_relax(mb_potential *pot, const char *evos_dir, int gen, int p0, int S, const int *nat, const int *atmn,
                  double *lat, double *x, double p_gpa, double urep, int rlxt, int mitr, double fmax, double *H,
                  int *iters, int *status);

/* Write one member's four files (no GPU needed): spcz[nspc] atomic numbers
 * of the species indices in atmn; lat0/x0 before and lat/x after relaxing
 * (Cartesian); H enthalpy and E energy (eV); frc[3N] and str[6] (virial, eV)
 * may be NULL; iters goes to OUTCAR's iteration line. */
int mb_evos_write(const char *evos_dir, int gen, int member, int N, int nspc, const int *spcz, const int *atmn,
                  const double *lat0, const double *x0, const double *lat, const double *x, double H, double E,
                  double p_gpa, const double *frc, const double *str, int iters);

/* RANK_TR's ranking (src/emod.c:304-393) of M members: order[k] = member
 * of rank k (lowest first, ties in member order) and, if fit != NULL, the
 * fitness fit[p] = (1 - tanh(2 (e_p - e_min) / (e_max - e_min) - 1)) / 2.
 * e_p = H[p] as the reference ranks (total enthalpy), or H[p] / nat[p]
 * with per_atom = 1 for populations of different sizes.  MB_ERR_STATE if
 * e_max - e_min < 1e-12 (the reference exits there). */
int mb_evos_rank(int M, const double *H, const int *nat, int per_atom, int *order, double *fit);

/* Per-species-pair radial distribution of S structures as RANK_TR's
 * duplicate test computes it (RDF, src/cell.c:369-417), on CUDA device
 * `device`: every (atom, image) pair within rmax with species(j) >=
 * species(i) adds exp(-(r - x_k)^2 / (2 sigma^2)) to the bins x_k = k rmax /
 * nbins within 3 sigma of r, times 1 below rmin and cos(pi/2 (x_k - rmin) /
 * (rmax - rmin)) above; same-species blocks halved; with normalise the whole
 * vector has unit length (RDF(C, 1)).  The reference uses nbins = 3000,
 * rmin 5.8, rmax 6.0, sigma 0.008 (src/util.c:1408-1410, src/cell.c:38).
 * Structures as mb_relax_batch (x Cartesian, ND periodic directions);
 * output rdf[S][nspc (nspc + 1) / 2][nbins], pairs m <= n row-major. */
int mb_rdf(int device, int S, const int *nat, const int *atmn, const double *lat, const double *x, int ND, int nspc,
           int nbins, double rmin, double rmax, double sigma, int normalise, double *rdf);

/* Overlaps of all pairs of S vectors of length len (CxC, src/cell.c:419-430,
 * for every pair of members at once): cxc[p*S + q] = sum_t rdf[p][t] rdf[q][t]. */
int mb_rdf_overlap(int device, int S, int len, const double *rdf, double *cxc);

/* RANK_TR's duplicate rule (src/emod.c:351-368) on M members in rank order:
 * for p from the worst up, the first better member k with COMP_CL(p, k) =
 * 0.8 cxc[p][k] + 0.1 exp(-(H_p - H_k)^2 / (2 0.05^2)) + 0.1 exp(-dv^2 /
 * (2 0.01^2)) > cut, dv = (V_p - V_k) / (2 (V_p + V_k)) (src/eutl.c:394-413),
 * marks p a duplicate: fit[p] *= 0.001 + (1 - COMP_CL)^2. */
int mb_evos_duplicates(int M, const double *cxc, const double *H, const double *vol, double cut, double *fit);

/* NVT molecular dynamics with the reference's thermostat (the RUNT == 2
 * branch of Dynamics, src/cmod.c:403-407, 440-453), entirely on the GPU:
 * per step  E+F+S -> K -> xi += dt/tau^2 (2K/(3 N T) - 1)
 *           -> x += v dt + f dt^2/2, v += f dt  (f = F/m - xi v) -> wrap.
 * v[3N] holds initial velocities (A/fs) and is updated; x (Cartesian) too.
 * T in K, dt in fs, tau = coupling time CPLT in fs.  If Hs/Ks are non-NULL
 * they receive H and K (eV) at the start of every step.  *xi carries the
 * thermostat variable in and out. */
int mb_md_nvt(mb_potential *pot, int N, int NM, int ND, const int *atmn, const double *lat9, double *x, double *v,
              double T, double dt, double tau, int nsteps, double urep, double *xi, double *Hs, double *Ks);

/* Maxwell initial velocities exactly as the reference draws them
 * (src/cmod.c:224-280) from its Park-Miller generator seeded by
 * PlantSeeds(seed) (src/util.c:1829-1873).  amu[N] are the atoms' masses
 * in atomic mass units; v[3N] receives velocities in Angstrom/fs for
 * temperature T (K).  Needs no GPU. */
int mb_maxwell(int N, const double *amu, double T, long seed, double *v);

/* Atomic mass (amu) of element z as tabulated by the reference (src/util.c:11). */
double mb_atomic_mass(int z);

/* Energy, forces and virial of one structure, like mb_efs, for callers that
 * cannot let the library allocate device memory: host codes that carve every
 * device buffer out of their own pre-sized pool or fixed memory budget, for
 * which a cudaMalloc inside their time-step loop could exceed the budget and
 * would synchronise the device under their streams.  This entry point has no
 * counterpart in the reference.  It allocates nothing: inputs and outputs are
 * the caller's device buffers, and all intermediates live in one fixed
 * device array of about 7.3 MB that every GPU loading the library holds
 * until the process exits.
 *   d_x[3N]   positions (Cartesian, device); read, not modified
 *   d_spc[N]  species (device)
 *   lat9      lattice (host)
 *   d_frc[3N] forces (device, written)
 *   d_out[8]  E, H, U[6] (device, written)
 * Limits: N <= 2048 atoms and at most 96 neighbours per atom; larger inputs
 * are rejected with MB_ERR_CAPACITY.  The work is queued on `stream` (a
 * cudaStream_t, 0 for the default stream) and the call returns once the
 * stream has run it (it reads back a 16-byte status word).  The first call
 * on a device looks up the array's device address with
 * cudaGetSymbolAddress; make that first call before any stream capture.
 * All calls share the one array and it keeps the last call's contents:
 * calls that overlap on the GPU (other streams, other host threads) race
 * and must not be issued. */
int mb_efs_noalloc(mb_potential *pot, int N, int NM, int ND, const double *lat9, const double *d_x, const int *d_spc,
                   double p_gpa, double urep, double *d_frc, double *d_out, void *stream);

/* ---- diagnostics (no counterpart in the reference) ---- */

/* Replay captured CUDA graphs (enable=1, the default; the environment
 * variable MAISE_B200_GRAPHS=0 makes 0 the default) or issue plain launches
 * (0).  Graphs are used for the NVT loop of mb_md_nvt (chunks of 10 steps)
 * and for every single-structure pass (mb_efs, mb_energy, CALL_MAISE and
 * each evaluation of mb_relax / mb_relax_fmax: wrap, list, descriptor pass,
 * finalize and the result copies in one launch, the cell updated in place).
 * A graph is captured once and replayed while the buffers and sizes it was
 * captured for hold; results are the same either way. */
int mb_graphs(mb_potential *p, int enable);

/* Start (enable=1) or stop timing of the fused descriptor/force kernel: every
 * launch is bracketed by CUDA events on the handle's stream (up to
 * `capacity` launches), and the kernel's pair/triplet counters are reset. */
/* The autotuner's decisions so far: *count (at most cap) entries; entry k
 * holds the pass mode (0 descriptors, 1 energy, 2 E/F/S, 3 VJP), whether the
 * leg-table kernel ran (legs), the size bucket (N <= 2^bucket), the
 * neighbour capacity, the chosen shape (warps per atom, atoms per CTA) and
 * the leg kernel's reverse-pass layout (0 per-lane runs of list entries,
 * 1 consecutive entries per round). */
int mb_tune_read(const mb_potential *pot, int cap, int *count, int *mode, int *legs, int *size_bucket, int *capacity,
                 int *wpa, int *apb, int *layout);
int mb_profile(mb_potential *pot, int enable, int capacity);

/* Synchronise and report: summed duration (ms) and number of timed launches
 * of the fused kernel, and the neighbour pairs and accepted triplets it
 * processed since mb_profile(pot, 1, ...). */
int mb_profile_read(mb_potential *pot, double *total_ms, int *launches, unsigned long long *pairs,
                    unsigned long long *triplets);

/* Time every step of mb_md_nvt with CUDA events (up to `capacity` steps)
 * and, if flush_bytes > 0, overwrite a scratch buffer of that size between
 * steps, outside the timed events, so that no step starts with the previous
 * step's data in L2.  enable = 0 turns both off. */
int mb_md_profile(mb_potential *pot, int enable, int capacity, size_t flush_bytes);

/* Summed step time (ms) and number of timed steps since mb_md_profile(pot, 1, ...). */
int mb_md_profile_read(mb_potential *pot, double *total_ms, int *steps);

/* Energy+gradient evaluations and kernel time (ms) of the last
 * mb_relax_batch call on this handle. */
int mb_batch_stats(const mb_potential *pot, long long *evals, double *ms);

/* Work of the last mb_relax_batch / mb_efs_batch launch: atom evaluations,
 * neighbour pairs and forward triplets summed over all evaluations (the
 * counts behind the batched kernel's FLOP rate). */
int mb_batch_work(const mb_potential *pot, long long *atom_evals, long long *pairs, long long *triplets);

/* Throughput of independent FP32 FMA chains filling every SM, TFLOP/s (the
 * FP32 roofline denominator of the batched relax). */
int mb_fp32_peak(int device, double *tflops);

/* Sustained FP64 FMA throughput of `device` in TFLOP/s, measured with an
 * FMA-chain kernel over every SM (a roofline denominator for FP64 work). */
int mb_fp64_peak(int device, double *tflops);

/* CUDA stream the handle launches on (a cudaStream_t), for callers that
 * time or order work around it. */
void *mb_stream(mb_potential *pot);

/* Number of kernel launches this handle has issued since it was opened. */
long mb_launch_count(const mb_potential *pot);

#ifdef __cplusplus
}
#endif
#endif
