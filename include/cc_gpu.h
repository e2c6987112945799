/* cc_gpu.h — C ABI of the B200 collective-coordinate (CC) potential library (libccgpu.so).
 *
 * The library evaluates, on one GPU, the stealthy collective-coordinate potential of a periodic point pattern:
 *   rho(k)   = sum_j exp(i k.r_j)                              over the constraint set {k, V(k)},
 *   Phi      = sum_k V(k) |rho(k)|^2 / Volume + Shift,
 *   F_j      = -dPhi/dr_j = (2/Volume) sum_k V(k) Im(conj(rho(k)) exp(i k.r_j)) k,
 *   S(k)     = |rho(k)|^2 / N.
 * Every k must lie on the reciprocal lattice of the cell: k = sum_e n_e b_e with integer n. Positions are given as
 * fractional (relative) coordinates s in the cell basis, r = sum_i s_i a_i, and wrapped into [0,1) the way the
 * reference's Configuration::Insert wraps them.
 *
 * Conventions: every call returns an int status (CC_OK = 0, negative on error); no exception crosses the ABI. Host
 * buffers are copied in and out; a handle owns its device buffers and one CUDA stream. Calls on one handle are not
 * thread-safe (as one reference potential object is not), distinct handles are independent.
 *
 * Reference interfaces replaced (paths within the reference project):
 *   cc_create / cc_create_cartesian   ShiftedCCPotential(dim) + constraints/AddConstraint + Shift
 *                                     (potential/CollectiveCoordinatePotential.h:84-117, :1318-1331)
 *   cc_set_positions                  ShiftedCCPotential::SetConfiguration (:1457-1463), which binds a Configuration
 *                                     built by Configuration::Insert (core/PeriodicCellList.h:517-538)
 *   cc_energy_grad                    Energy() then AllForce() (:1351-1372, :1434-1448), i.e. the bitwise contract of
 *                                     CombinedEnergyForce::EnergyAndAllForce (potential/CombinedEnergyForce.h)
 *   cc_rho                            GetRho() / RhoReal, RhoImag (:1255-1314)
 *   cc_force_one                      Force(result, i) (:1377-1394)
 *   cc_structure_factor               StructureFactor(config, k) (pairstat/StructureFactor.cpp:56-65)
 *   cc_objective                      Objective, Switch 0 (potential/StructureOptimization.cpp:447-536)
 */
#ifndef CC_GPU_H
#define CC_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
	CC_OK = 0,
	CC_ERR_ARG = -1,          /* invalid argument (null pointer, bad size, dimension outside 1..3, NaN input) */
	CC_ERR_OOM = -2,          /* device or host allocation failed */
	CC_ERR_CUDA = -3,         /* a CUDA call failed; cc_last_error() has the message */
	CC_ERR_TIMEOUT = -4,      /* a bounded device wait ran out */
	CC_ERR_NONLATTICE = -5,   /* a Cartesian k is not on the reciprocal lattice of the cell */
	CC_ERR_STATE = -6,        /* call order: e.g. energy requested before positions were set */
	CC_ERR_NOGPU = -7,        /* no CUDA device is visible: the library has no CPU path */
	CC_ERR_NAN = -8           /* cc_objective: the first variable is NaN (the reference's NotANumberFound) */
};

enum {
	CC_PREC_FP64 = 0,   /* FP64 seeds, FP64 recurrences, FP64 sums */
	CC_PREC_MIXED = 1   /* FP64 argument reduction, FP32 seeds and recurrences, FP64 tile partials and sums */
};

typedef struct cc_handle cc_handle;

/* Message of the last failed call on this thread (static storage, never NULL). */
const char *cc_last_error(void);

/* 1 if a CUDA device is usable, 0 otherwise. */
int cc_device_available(void);

/* Create a potential. d in 1..3; basis: d rows of d doubles, row i = basis vector a_i of the cell;
 * modes: M x d integers n (k = sum_e n_e b_e, b the reciprocal basis, b_e . a_i = 2 pi delta_ei); V: M weights;
 * shift: added to the energy. Modes may repeat, be zero or negative, in any order. M may be 0. */
int cc_create(int d, const double *basis, int64_t M, const int32_t *modes, const double *V, double shift,
              cc_handle **out);

/* As cc_create with Cartesian k (M x d). Each k is mapped to n_e = k.a_e / (2 pi); CC_ERR_NONLATTICE if some n_e is
 * not within 1e-9 (relative to max(1,|n_e|)) of an integer. */
int cc_create_cartesian(int d, const double *basis, int64_t M, const double *k, const double *V, double shift,
                        cc_handle **out);

/* The S2 form, the reference's ShiftedCCPotential_S2 (potential/CollectiveCoordinatePotential.h:1642-1749, constraints
 * added by its AddConstraint(k, {V, S0})): E = sum_m V_m (|rho(k_m)|^2 / N - S0_m)^2 + shift, with no volume factor,
 * F_i = (4 / N) sum_m V_m (|rho|^2 / N - S0_m) Im(conj(rho) e^{i k.r_i}) k_m. Arguments as cc_create plus S0 (M
 * targets); a repeated mode is one slot with the weights summed, the weighted mean target and the rest of the sum
 * in the shift (CC_ERR_ARG when its weights sum to zero but are not all zero). Evaluated in FP64 on the split rho / reduce / force path
 * whatever the precision asked; cc_set_path(CC_PATH_NUFFT), single-particle moves and batches refuse it (CC_ERR_ARG). */
int cc_create_s2(int d, const double *basis, int64_t M, const int32_t *modes, const double *V, const double *S0,
                 double shift, cc_handle **out);

/* The S2 form over nsub sub-configurations, the reference's ShiftedCCPotential_S2_MultiConfig
 * (potential/CollectiveCoordinatePotential.h:1756-1870): particles [c Np, (c + 1) Np), Np = N / nsub, form
 * sub-configuration c; E = sum_m V_m (<S(k_m)> - S0_m)^2 + shift with <S> = sum_c |rho_c|^2 / (Np nsub), and the
 * force on a particle of sub-configuration c is (4 / (Np nsub)) sum_m V_m dS_m Im(conj(rho_c) e^{i k.r}) k_m. N must
 * be a multiple of nsub (CC_ERR_ARG otherwise); cc_rho refuses the handle (rho is per sub-configuration). Otherwise as
 * cc_create_s2; nsub = 1 is the S2 form. */
int cc_create_s2_multiconfig(int d, const double *basis, int64_t M, const int32_t *modes, const double *V,
                             const double *S0, double shift, int nsub, cc_handle **out);

/* The sub-configuration count of an S2 handle (cc_create_s2 / cc_create_s2_cartesian): nsub > 1 makes it the
 * multi-configuration form of cc_create_s2_multiconfig, 1 the S2 form. CC_ERR_ARG for a plain handle with
 * constraints, nsub < 1, or bound positions whose count is not a multiple of nsub. */
int cc_set_subconfigurations(cc_handle *h, int nsub);

/* As cc_create_s2 with Cartesian k (M x d), mapped to modes as in cc_create_cartesian. */
int cc_create_s2_cartesian(int d, const double *basis, int64_t M, const double *k, const double *V, const double *S0,
                           double shift, cc_handle **out);

int cc_destroy(cc_handle *h);

/* Number of constraints, dimension, volume and the integer modes (M x d) of a handle. */
int cc_info(const cc_handle *h, int64_t *M, int *d, double *volume, int32_t *modes);

/* Real offset added to every Re rho(k) (the reference's HAVETWOFIXEDPARTICLES build adds 2). Default 0. */
int cc_set_rho_offset(cc_handle *h, double offset);

/* Bind N particles at fractional coordinates frac (N x d, host). N may be 0. */
int cc_set_positions(cc_handle *h, int64_t N, const double *frac);

/* Energy and Cartesian forces (N x d, host; F may be NULL) of the bound positions. precision: CC_PREC_*. */
int cc_energy_grad(cc_handle *h, double *E, double *F, int precision);

/* rho(k) of the bound positions in constraint order (host arrays of M). */
int cc_rho(cc_handle *h, double *re, double *im, int precision);

/* Force on particle i of the bound positions (d doubles), from the last cc_energy_grad. */
int cc_force_one(cc_handle *h, int64_t i, double *f);

/* S(k) = |rho(k)|^2 / N of the bound positions at K integer modes (K x d), host output S (K). */
int cc_structure_factor(cc_handle *h, int64_t K, const int32_t *modes, double *S, int precision);

/* The structure optimiser's Switch-0 objective: x = rescale * fractional coordinates (N*d), returns the energy in
 * *f and, if grad is not NULL, grad[i*d+j] = -F_i . a_j / rescale. A NaN first variable returns CC_ERR_NAN and
 * leaves *f and grad untouched, where the reference's Objective throws NotANumberFound
 * (potential/StructureOptimization.cpp:460-461; its catch at :571 takes InvalidStructure only); any other non-finite
 * variable returns CC_ERR_ARG. */
int cc_objective(cc_handle *h, int64_t N, const double *x, double rescale, double *f, double *grad, int precision);

/* --- structure optimisation (L-BFGS on the device) --------------------------------------------------------------
 * Replaces the structure optimiser's L-BFGS loop (RelaxStructure_NLOPT / _inner / _Emin,
 * potential/StructureOptimization.cpp:881-1090, with NLopt's or LuksanPLIS's L-BFGS, potential/LuksanPLIS.cpp:1668-)
 * for the Switch-0 objective (particle coordinates only). The variables are the fractional coordinates; positions,
 * gradient, the m correction pairs and every dot product stay on the device (FP64). The method is L-BFGS in the compact
 * representation (Byrd, Nocedal & Schnabel 1994) with Armijo backtracking; iterates are not NLopt's bit for bit. */
enum {
	CC_PREC_SCHEDULE = 2        /* cc_minimize: mixed precision until E/N <= switch_energy_per_particle, then FP64 */
};
#define CC_STOPVAL_GROUND_STATE (-1.0)
typedef struct {
	int history;                /* correction pairs m (1..64), default 40 as the reference's LBFGSHistory */
	int64_t max_evals;          /* evaluation limit, default 100000 */
	double stopval;             /* stop when E <= stopval, default -1e300; CC_STOPVAL_GROUND_STATE: E <= 1e-20 N */
	double gtol;                /* stop when max |dE/ds| <= gtol, default 0 */
	double ftol;                /* stop after 3 accepted steps with E decreasing by <= ftol |E|, default 1e-15 */
	int precision;              /* CC_PREC_FP64 (default), CC_PREC_MIXED or CC_PREC_SCHEDULE */
	double switch_energy_per_particle;   /* CC_PREC_SCHEDULE threshold, default 1e-12 */
	int iters_per_check;        /* iterations per host status check (one CUDA graph replay), default 32 */
} cc_lbfgs_opts;

typedef struct {
	double E;                   /* FP64 energy of the returned configuration */
	int64_t evals, iters;
	int status;                 /* 1 stop value, 2 gradient, 3 evaluation limit, 4 line search, 5 relative change */
} cc_lbfgs_result;

int cc_lbfgs_defaults(cc_lbfgs_opts *opts);

/* Minimise the energy from the fractional start frac (N x d, host), which receives the result wrapped into [0,1).
 * The handle's bound positions become the result. */
int cc_minimize(cc_handle *h, int64_t N, double *frac, const cc_lbfgs_opts *opts, cc_lbfgs_result *result);

/* --- batches of independent configurations (no counterpart in the reference, which evaluates one at a time) ---
 * A batch holds `count` instances, each an existing handle (its cell, constraint set, Shift) with a fixed particle
 * count N[i]. One evaluation of the batch is ONE persistent launch of the fused batch kernel: the rho, split-reduction
 * and force work items of every instance, of every dimension, share one work queue, an instance's phases ordered by
 * completion counts (bounded waits: CC_ERR_TIMEOUT if one runs out); a batched minimisation runs every instance's
 * L-BFGS at once, and instances that have finished are skipped item by item. An instance's results do not depend on
 * the rest of the batch. The handles must outlive the batch. */
typedef struct cc_batch cc_batch;
int cc_batch_create(int count, cc_handle *const *handles, const int64_t *N, cc_batch **out);
int cc_batch_destroy(cc_batch *b);
/* Bind positions (host, frac[i] is N[i] x d_i) to the batch's device buffers. */
int cc_batch_set_positions(cc_batch *b, const double *const *frac);
/* Evaluate every instance at its bound positions: energies E[count] and, if F is not NULL, forces F[i] (host). */
int cc_batch_energy_grad(cc_batch *b, double *E, double *const *F, int precision);
/* The same, enqueued on `stream` with results left on the device (no host synchronisation). */
int cc_batch_eval_device(cc_batch *b, int precision, void *stream);
/* Minimise every instance from its bound positions; frac[i] (host) receives the results, results[i] the outcomes. */
int cc_batch_minimize(cc_batch *b, double *const *frac, const cc_lbfgs_opts *opts, cc_lbfgs_result *results);
/* Autotuner of the batch's tile shapes: times `reps` FP64 evaluations of the bound positions for every candidate
 * (particles per rho block 32 / 64 / 128 / 256 / 512 / 1024 x segments per force block 32 / 64 / 128 / 256 / 512 /
 * 1024) with CUDA events and keeps the fastest for the batch's later evaluations and minimisations (default before
 * tuning: 64 x 64). The chosen shape
 * is returned in *per_split and *segs_per_split (either may be NULL). Results of different shapes agree to rounding;
 * with one shape every instance's result is independent of the rest of the batch. */
int cc_batch_autotune(cc_batch *b, int reps, int *per_split, int *segs_per_split);
/* Test hook of the fused batch kernel's bounded waits: every wait gives up after `polls` polls (0: the default, about
 * half a second) and, with phantom > 0, the reduction items of the first instance in the launch order wait for
 * `phantom` rho items more than it has, so their waits run out: the evaluation then returns CC_ERR_TIMEOUT (its
 * results are not to be used) and clears the error, and the next evaluation with phantom = 0 is a normal one. */
int cc_batch_set_wait_test(cc_batch *b, unsigned polls, int phantom);

/* --- Monte Carlo moves ----------------------------------------------------------------------------------------------
 * Replace ShiftedCCPotential_ForMC::TryMove / AcceptMove (potential/CollectiveCoordinatePotential.h:1906-1957): the
 * energy change when one particle moves from s_prev to s_after (fractional coordinates, d doubles each), in O(M)
 * from rho(k) of the bound positions, which the first call computes and AcceptMove then keeps current. The handle's
 * bound positions are not changed (the caller moves its particle, as the reference's MC drivers do).
 * AcceptMove without a pending trial returns CC_ERR_STATE. */
int cc_mc_try_move(cc_handle *h, const double *s_prev, const double *s_after, double *dE);
int cc_mc_accept_move(cc_handle *h);

/* --- ground-state server with continuous batching (no counterpart in the reference) ------------------------------
 * Each request is a stealthy configuration in a periodic cube of unit density (side N^(1/d)): the CLI's k-set for
 * (d, N, chi) with weights vtype (0: v = 1, 3: v = (1 - |k|/K)^2, as cc_kset_stealthy), a start frac0 (N x d) and an
 * arrival time in seconds after the call starts. The server minimises every request to Phi/N < 1e-20 (FP64), admitting
 * arrived requests while a slot is free and their device memory fits hbm_budget, and running all admitted requests
 * together, iters_per_round L-BFGS iterations per round; finished requests leave between rounds.
 * Admission scans the arrived requests in arrival order and admits each one that fits, so a large request waiting for
 * memory does not hold back smaller ones behind it, until it has waited max_bypass_s (then nothing behind it is
 * admitted before it). A request that cannot be served is rejected on its own and the others carry on: its result
 * has status CC_ERR_ARG (invalid request, e.g. d outside 1..3, N < 1, chi <= 0, an empty k-set), CC_ERR_OOM (its
 * estimated memory exceeds hbm_budget, or the pool could not allocate it) or CC_ERR_CUDA (its set-up copies failed),
 * E = NaN, evals = 0 and t_admit = t_done = the time of the rejection. cc_serve itself returns an error only when
 * the server cannot run at all (no device, invalid options, a failed launch). */
typedef struct {
	int d;
	int64_t N;
	double chi;
	int vtype;
	const double *frac0;
	double arrival_s;
	int64_t max_evals;          /* 0: 100000 */
	double *frac_out;           /* if not NULL: receives the final positions (N x d fractional) when the request ends */
} cc_request;
typedef struct {
	double E;                   /* energy at the end (FP64) */
	int64_t evals;
	int status;                 /* as cc_lbfgs_result.status (1..5), or a negative CC_ERR_* for a rejected request */
	double t_admit, t_done;     /* seconds after the call started */
} cc_request_result;
typedef struct {
	size_t hbm_budget;          /* bytes for the admitted requests, default 16 GiB */
	int max_slots;              /* admitted requests at most, default 256 */
	int iters_per_round;        /* default 16 */
	int history;                /* L-BFGS pairs, default 40 */
	double max_bypass_s;        /* admission may pass a waiting request for this long, default 1 s; 0: strict order */
} cc_serve_opts;
int cc_serve(const cc_request *reqs, int count, const cc_serve_opts *opts, cc_request_result *results, double *wall_s);
const char *cc_serve_last_error(void);

/* Many configurations from host memory in one call: frac (P x N x d fractional coordinates, host), E (P energies,
 * host) and F (P x N x d Cartesian forces, host, may be NULL). The same results, bitwise, as P calls of
 * cc_set_positions + cc_energy_grad (coordinates outside [0,1) are wrapped the same way; a non-finite one fails the
 * call with CC_ERR_ARG). The positions go to the device in chunks of 64 configurations on a second stream while
 * earlier chunks are evaluated, and the evaluations follow one another without host synchronisation (each rho kernel
 * overlaps the previous evaluation's force kernel); pinned host buffers (cudaHostAlloc, cudaHostRegister) let the
 * copies overlap. The call returns when E and F are written. Every configuration of a call is resident on the
 * device at once (2 P N d doubles). Replaces a loop of the reference's SetConfiguration + Energy + AllForce over
 * configurations (potential/CollectiveCoordinatePotential.h:1351-1448). */
int cc_energy_grad_many(cc_handle *h, int64_t P, int64_t N, const double *frac, double *E, double *F, int precision);

/* Device-resident evaluation: d_frac (N x d, device), outputs d_E (1 double) and d_F (N x d Cartesian, may be
 * NULL) and d_gfrac (N x d gradient of the energy with respect to the fractional coordinates, may be NULL), all on
 * the device, enqueued on `stream` (a cudaStream_t; NULL = the handle's stream). No host synchronisation. */
int cc_energy_grad_device(cc_handle *h, int64_t N, const double *d_frac, double *d_E, double *d_F, double *d_gfrac,
                          int precision, void *stream);

/* Generate the stealthy k-set of the reference's CLI (GeneratePotential Type 0..3): the half-space reciprocal
 * vectors (first nonzero index > 0) sorted by |k|, the first ceil(chi*N*d) of them plus the rest of the last shell;
 * V = 1 (type 0), acos(x)-x*sqrt(1-x^2) (1), (1-x)^6 (2), (1-x)^2 (3) with x = |k|/K, K the first excluded |k|.
 * Writes at most cap modes; *M receives the count (CC_ERR_ARG if cap is too small, *M then holds the need). */
int cc_kset_stealthy(int d, const double *basis, int64_t N, double chi, int type, int64_t cap, int32_t *modes,
                     double *V, int64_t *M);

/* --- isotropic structure factor ---------------------------------------------------------------------------------
 * cc_kset_isotropic: the wavevectors of GetKs (core/PeriodicCellList.cpp:509-735) for a cell (host only, no GPU
 * needed), as K integer modes (K x d) with |k| (K): for d >= 2 the half-space lattice points with
 * circular_kmin < |k| < circular_kmax ordered by (|k|^2, k_x), or, when linear_kmax differs from circular_kmax, the
 * multiples i k (|i k| <= linear_kmax) of the first point of each lattice direction in that circle; for d = 1 the
 * multiples of the reciprocal vector (see the reference for circular_kmin > 0). sample_probability < 1 keeps each
 * multiple with that probability, drawn as the reference draws it (Mersenne Twister seeded with 98765).
 * *K receives the count (CC_ERR_ARG if cap is too small, *K then holds the need).
 *
 * cc_isotropic_structure_factor: IsotropicStructureFactor (pairstat/StructureFactor.cpp:79-260) over nconfigs
 * configurations (bases: nconfigs x d x d, row i = a_i; N[j] particles at frac[j], N[j] x d fractional): S(k) of every
 * wavevector on the GPU (FP64), binned by floor(|k| / k_precision) (k_precision 0: the first reciprocal vector's
 * length). option 0: bin means over wavevectors; 1: S(k) averaged over the k-space shell volume for |k| <=
 * circular_kmax; 2: one row per wavevector (every cell must give the same count), sorted by |k|. Rows of 4 doubles
 * (k, S, dk, dS) as the reference's GeometryVector(4) results; *count receives the number of rows (CC_ERR_ARG if cap
 * is too small). Wavevectors are recomputed when a configuration's basis differs from the previous one. */
int cc_kset_isotropic(int d, const double *basis, double circular_kmax, double linear_kmax, double sample_probability,
                      double circular_kmin, int64_t cap, int32_t *modes, double *kamp, int64_t *K);
int cc_isotropic_structure_factor(int d, int64_t nconfigs, const double *bases, const int64_t *N,
                                  const double *const *frac, double circular_kmax, double linear_kmax,
                                  double k_precision, double sample_probability, int option, double circular_kmin,
                                  double *results, int64_t cap, int64_t *count);

/* --- multi-species stealthy potential with soft-core contact -----------------------------------------------------
 * MultiStealthyPotential (apps/CCOptimization/MultiStealthyPotential.h:115-481, .cpp:139-985):
 *   E   = u0 sum_s (N_s/N) Phi_s + e0 sum_{i<j} sum_images [r < s_ij] (1 - r/s_ij)^2,   s_ij = R_i + R_j,
 *   F_i = u0 (N_s/N) F_i^(CC,s) + e0 sum_{j != i} sum_images [r < s_ij] (2/s_ij)(1/r - 1/s_ij)(r_i - r_j),
 * Phi_s the collective-coordinate energy of species s over its own particles (constraint set: M[s] integer modes
 * modes[s] (M[s] x d) with weights V[s]); coincident particles (r < 1e-15) get the reference's unit push along the
 * first axis. The contact term is off when |e0| <= 1e-10 (as the reference's WithRepulsion).
 * cc_multi_set_configuration: N particles at fractional frac (N x d), species[i] in 0..nspecies-1, radii (N, each
 * > 0) or NULL for the reference's default 0.5. cc_multi_energy_grad: E and, if F is not NULL, Cartesian forces
 * (N x d). Calls on one object are not thread-safe. */
typedef struct cc_multi cc_multi;
int cc_multi_create(int d, const double *basis, int nspecies, const int64_t *M, const int32_t *const *modes,
                    const double *const *V, double u0, double e0, cc_multi **out);
/* As cc_multi_create with S0[s] (M[s] targets) making species s's Phi_s the S2 form (cc_create_s2);
 * a NULL S0[s] keeps that species plain. With one species, u0 = 1 and radii sigma / 2 this is the reference's
 * RepulsiveCCPotential (apps/CCOptimization/RepulsiveCCPotential.h:21-159) with an S2 kernel (S0 != 0). */
int cc_multi_create_s2(int d, const double *basis, int nspecies, const int64_t *M, const int32_t *const *modes,
                       const double *const *V, const double *const *S0, double u0, double e0, cc_multi **out);
int cc_multi_set_configuration(cc_multi *m, int64_t N, const double *frac, const int32_t *species,
                               const double *radii);
int cc_multi_energy_grad(cc_multi *m, double *E, double *F);
int cc_multi_destroy(cc_multi *m);

/* --- allocation-free evaluation (no counterpart in the reference) -----------------------------------------------
 * For callers that cannot allocate GPU memory: processes whose memory manager (a caching allocator, a serving
 * engine with a fixed HBM budget) owns the device's memory and lets no library allocate beside it, and loops that
 * must not pay for cudaMalloc, which can synchronise the device. They cannot create a cc_handle (cc_create
 * allocates). cc_energy_noalloc allocates nothing, on the device or the host: the caller passes
 * every input and output in its own device memory, and the only scratch is a fixed array of
 * CC_NOALLOC_SCRATCH_BYTES inside the library, which every GPU that loads the library holds until the process exits.
 *   d, basis (host, d x d), M modes (device, M x d int32), V (device, M), shift, N fractional positions (device,
 *   N x d); outputs: d_E (device, 1 double) = sum_m V_m |rho_m|^2 / volume + shift and, if not NULL, d_rho (device,
 *   M complex doubles as re,im pairs) in mode order. Work is enqueued on `stream` (cudaStream_t, NULL = legacy).
 * Limits: M <= CC_NOALLOC_MAX_MODES, N <= CC_NOALLOC_MAX_PARTICLES, else CC_ERR_ARG (see cc_noalloc_last_error).
 * The first call on each device looks up the scratch array's device address (and may load the kernel), so make it
 * before any stream capture, with that device current. All calls share the one scratch array and each call leaves
 * its contents behind (the call clears what must start at zero): calls whose work overlaps on the GPU, e.g. on
 * two streams at once, race and must be serialised by the caller. The looked-up address is kept per device for the
 * life of the process: after a cudaDeviceReset the next call would pass a stale address, so do not reset a device
 * between calls. */
#define CC_NOALLOC_SCRATCH_BYTES (16u << 20)
#define CC_NOALLOC_MAX_MODES 262144
#define CC_NOALLOC_MAX_PARTICLES (1 << 30)
int cc_energy_noalloc(int d, const double *basis, int64_t M, const int32_t *d_modes, const double *d_V, double shift,
                      int64_t N, const double *d_frac, double *d_E, double *d_rho, void *stream);
const char *cc_noalloc_last_error(void);

/* --- execution path (no counterpart in the reference) ---------------------------------------------------------
 * CC_PATH_SPLIT: three kernels per evaluation (rho, split reduction + energy, forces) chained by
 * programmatic dependent launch (value 1 is not a path: a cooperative one-kernel evaluation measured slower than the
 * split path at every size, 41.6 against 25.6 us at 3D N=2000, and was removed). CC_PATH_NUFFT: energies and forces by non-uniform FFTs (the reference's FINUFFT
 * backend, CollectiveCoordinatePotential.h:119-1250): a type-1 transform for rho, type-2 transforms for the forces,
 * "exponential of semicircle" kernel of width 14 on a fine grid of twice the mode range, always in FP64, errors
 * ~1e-13 of sum |c|; its cost grows with N w^d + grid log(grid) instead of N M, so it wins for many particles and
 * many modes. CC_PATH_AUTO (the default, as the reference gates its FINUFFT backend): the NUFFT path for an
 * evaluation whose estimated time is lower there (e.g. 2D N=1e5 with M=4e4 modes), the split path otherwise.
 * Results agree to rounding; each path repeats bitwise. */
enum { CC_PATH_SPLIT = 0, CC_PATH_NUFFT = 2, CC_PATH_AUTO = 3 };
int cc_set_path(cc_handle *h, int path);
/* The path (CC_PATH_SPLIT or CC_PATH_NUFFT) an evaluation of N particles at `precision` takes on this
 * handle under its current cc_set_path choice. */
int cc_eval_path(cc_handle *h, int64_t N, int precision, int *path);

/* on = 1: the caller promises that the positions given to cc_energy_grad_device on this handle were complete before
 * the kernel enqueued just before the call on its stream, and that no work in flight writes them (for example a pool
 * of resident configurations evaluated one after another). The rho kernel of such an evaluation then runs its
 * tables and phase sums while the previous kernel on the stream drains, and waits for that kernel only before it
 * writes its partial rows. Results are bitwise those of on = 0 (the default, for positions that a kernel just before
 * the call produced, such as an optimiser's update). Only the split path's rho kernel of cc_energy_grad_device
 * uses it; every other entry point ignores it. No counterpart in the reference (one evaluation per call there). */
int cc_set_independent_positions(cc_handle *h, int on);

/* Synchronise the device and report a CUDA error of an earlier device-path evaluation (no kernel of a handle waits
 * on another block, so there is no timeout to report here). */
int cc_check_device_error(cc_handle *h);

/* --- measurement support (no counterpart in the reference) --------------------------------------------------- */

/* on = 1: every following evaluation on this handle records CUDA events around its rho, reduce and force kernels
 * (on the stream they run on), also inside a stream capture (the events become graph nodes); cc_get_timing
 * synchronises and returns the summed kernel times in ms and the number of evaluations timed since timing was
 * switched on, then clears the record. Switching timing off keeps the record. */
int cc_set_timing(cc_handle *h, int on);
int cc_get_timing(cc_handle *h, double *rho_ms, double *reduce_ms, double *force_ms, int64_t *evals);

/* Launch configuration chosen for N particles: the rho kernel's particle splits and the force kernel's unit
 * splits, the segment length L and the number of segments (for reports). */
int cc_plan_info(const cc_handle *h, int64_t N, int *L, int64_t *nseg, int *nsplit, int *nksplit);

/* Measure the device's FMA throughput (TFLOP/s, 2 flops per FMA) of independent FMA chains in FP64
 * (precision = CC_PREC_FP64) or FP32 (CC_PREC_MIXED), timed with CUDA events: the roofline peak of this path. */
int cc_probe_fma_peak(int precision, double *tflops);

#ifdef __cplusplus
}
#endif

#endif /* CC_GPU_H */
