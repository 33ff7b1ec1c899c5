/*
 * cqg.h — C ABI of the B200 Monte Carlo wave-function (MCWF) ensemble engine.
 *
 * The engine replaces C++QED's EnsembleMCWF / MCWF_Trajectory hot path.  The
 * reference evaluates its quantum system through virtual callbacks
 * (structure::Hamiltonian::addContribution, Liouvillean::rates / actWithJ,
 * Averaged::average, Exact::actWithU) that cannot run on a GPU, so the system
 * is lowered ONCE on the host into the plain descriptor below (banded
 * "Tridiagonal" terms placed on tensor-product axes, jump operators with their
 * closed-form rates, linear observables) and every trajectory step then runs
 * on the device.
 *
 * Conventions
 *  - Complex numbers are two doubles {re, im}; layout-compatible with
 *    std::complex<double> and double2.
 *  - State vectors are C-order (last axis contiguous), as Blitz CArray<RANK>
 *    in the reference (quantumdata/Types.h:11-12).
 *  - Every function returns 0 on success or a negative CQG_E_* code; the
 *    message is available from cqg_last_error() (thread-local).
 *  - Handles are not thread-safe; distinct handles are independent.
 */
#ifndef CQG_H_INCLUDED
#define CQG_H_INCLUDED

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CQG_MAX_RANK 8
#define CQG_ABI_VERSION 5

/* ---- status codes ------------------------------------------------------ */
#define CQG_OK 0
#define CQG_E_INVALID (-1)       /* bad argument / inconsistent descriptor       */
#define CQG_E_CUDA (-2)          /* CUDA runtime error                            */
#define CQG_E_NOMEM (-3)         /* allocation failed / HBM budget exceeded       */
#define CQG_E_UNSUPPORTED (-4)   /* descriptor outside what the kernels handle   */
#define CQG_E_NONFINITE (-5)     /* a trajectory produced a non-finite value      */
#define CQG_E_STALLED (-6)       /* a trajectory exhausted its attempt budget     */
#define CQG_E_NODEVICE (-7)      /* no CUDA device / extension not usable         */

/* per-trajectory status bits (cqg_ensemble_status) */
#define CQG_TRAJ_NONFINITE_NORM 1u   /* MCWF_Trajectory.h:338 "Infinite detected"   */
#define CQG_TRAJ_NONFINITE_RATE 2u   /* LiouvilleanAveragedCommon.h:87-89           */
#define CQG_TRAJ_DT_UNDERFLOW 4u     /* step size collapsed below 1e-300 * t scale  */
#define CQG_TRAJ_ATTEMPT_LIMIT 8u    /* bounded retry loop gave up                  */

typedef struct cqg_complex {
  double re, im;
} cqg_complex;

/* ---- system descriptor ---------------------------------------------------
 * A banded operator in the sense of quantumoperator::Tridiagonal<RANK>
 * (quantumoperator/Tridiagonal.h:71-287) placed on `rank` axes of the system.
 * diagonal index  j = sum_a digit_a * 3^(rank-1-a)   (axis 0 most significant)
 *   digit 0: main diagonal      out n   <- in n      extent N_a
 *   digit 1: "minus" diagonal   out n+K <- in n      extent N_a-K_a
 *   digit 2: "plus"  diagonal   out n   <- in n+K    extent N_a-K_a
 * (Tridiagonal.tcc:220-263, ranges filled at :199-210).  Each diagonal is
 * NULL (empty) or a C-order array over its box.  `freqs` (NULL, or 3^rank
 * entries each NULL or box-shaped) gives the interaction-picture frequencies:
 * at picture time tau the coefficient is diagonal * exp(tau * freq)
 * (Tridiagonal::propagate, Tridiagonal.tcc:153-163).                       */
typedef struct cqg_tridiagonal {
  int32_t rank;
  int32_t axes[CQG_MAX_RANK];
  int64_t differences[CQG_MAX_RANK];
  const cqg_complex* const* diagonals;
  const cqg_complex* const* freqs;
} cqg_tridiagonal;

/* A jump operator J_m (structure::Liouvillean<RANK>::actWithJ, Liouvillean.h:54-60)
 * with its rate rule.  If rate_weights != NULL the rate is the closed form
 * sum_n rate_weights[n_axis] |psi_n|^2 over the normalised state (the
 * reference's element `rate` functions, e.g. 2 kappa <n>, Mode_.h:180-184);
 * otherwise the rate is ||J psi||^2 and the jump uses the normalised J psi
 * (the "special jump" convention, MCWF_Trajectory.h:279-291).             */
typedef struct cqg_jump {
  cqg_tridiagonal op;
  int32_t rate_axis;
  const double* rate_weights;
} cqg_jump;

/* An observable column source: Re or Im of <psi|O|psi> (linear in rho, as
 * structure::Averaged::average_v).  O is either a banded term (`dense` NULL)
 * or a dense N_axis x N_axis row-major matrix acting on `dense_axis`.     */
typedef struct cqg_observable {
  cqg_tridiagonal op;
  const cqg_complex* dense;
  int32_t dense_axis;
  int32_t col_re; /* output column of Re<O>, or -1 */
  int32_t col_im; /* output column of Im<O>, or -1 */
  /* fourier != 0 (with a dense matrix on dense_axis that is this same operator): the
   * observable is also given as the sum over the 1-D slices along dense_axis of
   * sum_x fourier_weights[x] |(F psi_slice)_x|^2, F the reference's k -> x transform
   * (quantumdata::ffTransform, LazyDensityOperatorFFT.cc:12-31), e.g. a particle's <X> and
   * <X^2> (Particle.cc:128-160).  The engine may then use a fast transform instead of the
   * dense matrix; the value is real (col_im must be -1). */
  int32_t fourier;
  int32_t reserved;
  const double* fourier_weights; /* [dims[dense_axis]] */
} cqg_observable;

/* The whole system: Hamiltonian terms H/i in the reference's application
 * order (frees in axis order, then interactions: BinarySystem.cc:194-207,
 * Composite.tcc:178-197), the Exact (interaction-picture) part as per-axis
 * exponents lambda_a[n] with U(tau) = prod_a exp(lambda_a[n_a] tau)
 * (FreeExact.h:31, Mode.cc:42-45), jumps in the reference's ordinal order,
 * and observables.                                                          */
typedef struct cqg_system_desc {
  int32_t rank;
  int64_t dims[CQG_MAX_RANK];
  int32_t n_ham;
  const cqg_tridiagonal* ham;
  int32_t has_hamiltonian;                    /* getHa() != nullptr            */
  const cqg_complex* exact[CQG_MAX_RANK];     /* NULL: axis has no Exact part  */
  int32_t n_jumps;
  const cqg_jump* jumps;
  int32_t n_obs;
  const cqg_observable* obs;
  int32_t n_avr;                              /* number of linear average columns */
  double highest_frequency;                   /* QuantumSystem::highestFrequency */
} cqg_system_desc;

/* ---- engine parameters (mcwf::Pars, ode_engine::Pars, randomutils::Pars) */
#define CQG_RNG_PCG64 0   /* pcg64{seed, prngStream+i}: MCWF_Trajectory.h:208,223-226 */
#define CQG_RNG_PHILOX 1  /* Philox4x32-10 keyed by seed, counter = (traj, draw)     */

#define CQG_FP64 0        /* complex128 state and operator                           */
#define CQG_FP32 1        /* complex64 state/operator; FP64 norm, error norm, dt, sums */

typedef struct cqg_mcwf_pars {
  double eps_rel;              /* --eps      (ODE.h:59) default 1e-6  */
  double eps_abs;              /* --epsAbs   (ODE.h:60) default 1e-12 */
  double dp_limit;             /* --dpLimit  (MCWF_Trajectory.h:41) 0.01 */
  double overshoot_tolerance;  /* --overshootTolerance (:42) 10 */
  double dt_init;              /* <= 0: 1/(10*highest_frequency) (Trajectory.h:126) */
  uint64_t seed;               /* --seed (Random.h:144) 1001 */
  uint64_t prng_stream;        /* --prngStream (Random.h:145) 1; trajectory i uses stream+i */
  int32_t rng;                 /* CQG_RNG_* */
  int32_t noise;               /* --noise: 0 switches the Liouvillean off (Structure.h:97-103) */
  int32_t precision;           /* CQG_FP64 / CQG_FP32 */
  int32_t max_attempts;        /* bounded ODE retries per step (0: default 100000) */
  int32_t autotune;            /* 1: time the candidate CTA shapes of each kernel group on a
                                  sample of its trajectories at creation and keep the fastest
                                  (cached per shape class and device); 0: fixed defaults */
  int32_t cta_threads;         /* > 0: force this CTA size on every group (no tuning); a
                                  multiple of 32, at most 128 for warp-per-trajectory groups
                                  and 512 for CTA-per-trajectory groups */
  int32_t cta_shared_vectors;  /* with cta_threads > 0, for CTA-per-trajectory groups: 1 keeps
                                  the stage derivatives in shared memory (when they fit), 0 in
                                  a global scratch slab; for warp-per-trajectory groups: 1 runs
                                  the instance compiled for more resident CTAs per SM (where
                                  there is one); the autotuner chooses otherwise */
  int32_t ip_phase_table;      /* interaction-picture phases exp(tau f) of the off-diagonal
                                  terms: 0 forms them once per distinct frequency f of the
                                  system (at most 128 on the warp kernel: per attempt, the
                                  stage powers of exp(dt f / 40); at most 1024 on the CTA
                                  kernel: per stage, bit-identical to -1), -1 forms them per
                                  row, slot and stage as the reference does */
  int32_t yield_steps;         /* warp-per-trajectory groups of more trajectories than the GPU
                                  holds at once: a warp hands its trajectory back to the work
                                  queue after this many MCWF steps and takes the next, so the
                                  end of a launch waits for one such chunk, not for whole
                                  trajectories; the results are bit-identical.  0: the default
                                  (64 for groups of Schroedinger-picture systems; groups with
                                  interaction-picture phases do not yield), > 0: every warp
                                  group, -1: never */
} cqg_mcwf_pars;

void cqg_mcwf_pars_default(cqg_mcwf_pars* p);

/* ---- errors / device --------------------------------------------------- */
const char* cqg_last_error(void);
int cqg_abi_version(void);
int cqg_device_count(int* count);

/* ---- systems ------------------------------------------------------------
 * Lower a descriptor to device memory.  Replaces the virtual plugin
 * interfaces structure::Hamiltonian/Liouvillean/Averaged/Exact
 * (Hamiltonian.h:38-43, Liouvillean.h:54-67, Averaged.h:37-49, Exact.h:58-61)
 * and quantumoperator::Tridiagonal::apply (Tridiagonal.tcc:220-233).      */
typedef struct cqg_system cqg_system;
int cqg_system_create(const cqg_system_desc* desc, cqg_system** out);
int cqg_system_dimension(const cqg_system* sys, int64_t* total_dim);
int cqg_system_destroy(cqg_system* sys);

/* Batched Hamiltonian::addContribution (Hamiltonian.h:38-43; the slice-wise
 * Tridiagonal::apply of the reference, Tridiagonal.tcc:220-263):
 *   dpsi_i += (H/i)(tau) psi_i,  i < n_states,  tau = t - t0 (interaction picture).
 * psi and dpsi are 16-byte aligned device pointers to n_states x D complex128 states,
 * state after state, and must not overlap (CQG_E_INVALID otherwise).  Queued on `stream` (a cudaStream_t, NULL = default stream);
 * returns without waiting. */
int cqg_system_apply_hamiltonian(const cqg_system* sys, const cqg_complex* psi, cqg_complex* dpsi, int64_t n_states,
                                 double tau, void* stream);

/* ---- ensembles ----------------------------------------------------------
 * mcwf::makeEnsemble (MCWF_Trajectory.h:213-234): n_traj copies of psi0
 * (sys dimension D complex values), trajectory i seeded with stream
 * prng_stream+i.  Trajectories may belong to different systems
 * (cqg_batch_create) — the uneven-batch case.                             */
typedef struct cqg_ensemble cqg_ensemble;
int cqg_ensemble_create(const cqg_system* sys, const cqg_complex* psi0, int64_t n_traj,
                        const cqg_mcwf_pars* pars, cqg_ensemble** out);

/* Batch of trajectories over several systems: trajectory i evolves
 * systems[sys_index[i]] from psi0s + psi0_offsets[i] (host pointer). */
int cqg_batch_create(const cqg_system* const* systems, int32_t n_systems, const int32_t* sys_index,
                     const cqg_complex* psi0s, const int64_t* psi0_offsets, int64_t n_traj,
                     const cqg_mcwf_pars* pars, cqg_ensemble** out);

/* Advance every trajectory by exactly Dt, n_intervals times (cppqedutils::advance,
 * Trajectory.h:44-50, inside Ensemble::advance, StochasticTrajectory.h:220).
 * After interval k the ensemble sums are written to avr_out[k*(n_avr+1) + c]
 * (host pointer, may be NULL): columns 0..n_avr-1 the linear averages, column
 * n_avr the dtDid — divide by n_traj for the ensemble mean; the reference streams
 * (1/N) Tr(rho O) and the mean dtDid (MCWF_Trajectory.h:406-420,
 * StochasticTrajectory.h:223-226).  In batch mode the columns of systems with
 * different observables are mixed; use cqg_ensemble_traj_averages instead.  */
int cqg_ensemble_run(cqg_ensemble* ens, double Dt, int32_t n_intervals, double* avr_out);

/* Same as cqg_ensemble_run but every trajectory advances to the absolute
 * time t_end (used for the T-capped final interval in Dt mode). */
int cqg_ensemble_advance_to(cqg_ensemble* ens, double t_end, double* avr_out);

/* `n_steps` MCWF steps per trajectory, each MCWF_Trajectory::step(T - t) (the
 * dc-mode loop of trajectory::run, Trajectory.h:560-595), stopping early at T.
 * n_steps = 0 only evaluates the averages of the current states. */
int cqg_ensemble_steps(cqg_ensemble* ens, int32_t n_steps, double T, double* avr_out);

/* Per-trajectory averages of the first output of the last run call:
 * out[i*(n_avr+1) + c], column n_avr = dtDid. */
int cqg_ensemble_traj_averages(cqg_ensemble* ens, double* out);

int cqg_ensemble_size(const cqg_ensemble* ens, int64_t* n_traj, int32_t* n_avr);
int cqg_ensemble_get_state(const cqg_ensemble* ens, int64_t i, cqg_complex* psi_out);
int cqg_ensemble_set_state(cqg_ensemble* ens, int64_t i, const cqg_complex* psi);

/* Scalars per trajectory (any pointer may be NULL): t, dtDid, dtTry. */
int cqg_ensemble_get_times(const cqg_ensemble* ens, double* t, double* dt_did, double* dt_try);

/* Logger counters per trajectory (MCWF_TrajectoryLogger.h:59-101, ODE.h:99-122):
 * counters[i*8 + k], k = 0 accepted steps, 1 ODE attempts, 2 failed ODE attempts,
 * 3 RHS evaluations, 4 dpLimit overshoots, 5 step-backs, 6 jumps, 7 status bits. */
int cqg_ensemble_get_counters(const cqg_ensemble* ens, uint64_t* counters);

/* Per trajectory (any pointer may be NULL): maximal dpLimit overshoot, maximal dpTolerance
 * overshoot and maximal |norm - 1| (mcwf::Logger, MCWF_TrajectoryLogger.cc:37-56). */
int cqg_ensemble_get_logger_maxima(const cqg_ensemble* ens, double* max_overshoot, double* max_tolerance_overshoot,
                                   double* max_norm_dev);

/* Jump record ring per trajectory: up to `cap` (time, lindblad) pairs of the
 * most recent jumps (MCWF logger jump list, MCWF_TrajectoryLogger.cc:42-75). */
int cqg_ensemble_get_jumps(const cqg_ensemble* ens, int64_t i, int32_t cap, double* times,
                           int32_t* lindblads, int32_t* n_out);

/* Every trajectory's jump ring at once, for a host that keeps all jump records (the ensemble
 * log's histogram of jump times, MCWF_TrajectoryLogger.cc:79-121): *cap (per-trajectory ring
 * capacity), counts[i] (jumps of trajectory i so far; its k-th jump is at slot k mod cap
 * while k >= counts[i] - cap), times and lindblads [n_traj][cap].  Any pointer may be NULL. */
int cqg_ensemble_get_jump_rings(const cqg_ensemble* ens, int32_t* cap, uint64_t* counts, double* times,
                                int32_t* lindblads);
/* Changes the per-trajectory ring capacity (default 64), keeping the most recent records.
 * A checkpoint loads only into an ensemble with the capacity it was saved with. */
int cqg_ensemble_set_jump_capacity(cqg_ensemble* ens, int32_t cap);

/* OR of all trajectory status bits; CQG_E_NONFINITE / CQG_E_STALLED when set. */
int cqg_ensemble_status(const cqg_ensemble* ens, uint32_t* bits);

/* Device times of the last run call in milliseconds (CUDA events on the
 * ensemble's stream): the MCWF kernel alone, and every device operation of the
 * call (initialisation, kernel, reduction, read-back).  Either pointer may be NULL. */
int cqg_ensemble_last_kernel_ms(const cqg_ensemble* ens, double* kernel_ms, double* run_ms);

/* Launch plan of an ensemble (no reference counterpart: the reference runs its
 * trajectories one after another).  Trajectories are grouped by kernel shape, each group
 * one persistent launch per run call, the groups on concurrent streams.  Writes the number
 * of groups to *n_groups and, for the first min(n_groups, cap) groups, five int32 each to
 * plan: kind (0 = warp per trajectory, 1 = CTA per trajectory with the stage derivatives in
 * global scratch, 2 = CTA per trajectory with them in shared memory, 3 = warp per trajectory
 * with the instance compiled for more resident CTAs per SM), rows per lane E (warp
 * kind), off-diagonal slot bound, CTA threads, trajectories in the group. */
int cqg_ensemble_plan(const cqg_ensemble* ens, int32_t* n_groups, int32_t* plan, int32_t cap);

/* ---- checkpoint / continuation -------------------------------------------
 * The role of the reference's trajectory state archive (trajectory::writeViaSStream /
 * readViaSStream, Trajectory.h:353-424, MCWF_Trajectory.h:134-147, used by --continue),
 * in this library's own binary layout: every trajectory's state vector, t, t0, dtTry,
 * dtDid, random stream, logger counters and maxima, status and jump records.
 * cqg_ensemble_save with buf == NULL or cap too small only reports the size.
 * cqg_ensemble_load requires an ensemble created over the same systems, trajectory
 * count and precision; the continued run is bit-identical to an uninterrupted one.      */
int cqg_ensemble_save(const cqg_ensemble* ens, void* buf, uint64_t cap, uint64_t* size);
int cqg_ensemble_load(cqg_ensemble* ens, const void* buf, uint64_t size);

/* ---- master equation ------------------------------------------------------
 * quantumtrajectory::Master (Master.h:153-208) on the device for the same system:
 * drho/dt = A rho + (A rho)^+ + sum_m J_m rho J_m^+ (A = H/i), the controlled Cash-Karp
 * step of the trajectories over all D^2 elements, then U rho U^+ with the exact part and
 * exact Hermiticity and normalisation.  rho starts as |psi0><psi0|.  Rows are the
 * expectation values Tr(O rho) of the system's n_avr linear averages followed by dtDid.
 * Memory: 11 D x D complex128 matrices.                                              */
typedef struct cqg_master cqg_master;
int cqg_master_create(const cqg_system* sys, const cqg_complex* psi0, const cqg_mcwf_pars* pars, cqg_master** out);
/* n_intervals intervals of Dt (ODE steps never cross an interval's end), one row each. */
int cqg_master_run(cqg_master* m, double Dt, int32_t n_intervals, double* avr_out);
/* Up to n_steps ODE steps of size T - t (dc mode), then one row (avr_out may be NULL). */
int cqg_master_steps(cqg_master* m, int32_t n_steps, double T, double* avr_out);
int cqg_master_averages(cqg_master* m, double* avr_out);
/* rho in row-major order (D x D complex128). */
int cqg_master_get_rho(const cqg_master* m, cqg_complex* rho);
int cqg_master_get_times(const cqg_master* m, double* t, double* dt_did, double* dt_try);
int cqg_master_destroy(cqg_master* m);

/* ---- request server ------------------------------------------------------
 * Continuous batching of ensemble requests (no reference counterpart: C++QED runs one
 * ensemble at a time, Ensemble::advance, StochasticTrajectory.h:220-245).  A request is a
 * system, an initial state, n_traj trajectories (pcg64 streams prng_stream + i, as in an
 * ensemble), an end time T and an output interval Dt; its result is one row of ensemble
 * sums per interval (the system's n_avr linear averages, then the dtDid column), exactly the
 * rows cqg_ensemble_run would give for the same request alone.  Each cqg_server_round
 * admits waiting requests in arrival order whose trajectories fit the free slots and whose
 * states fit the free state heap (hbm_budget_bytes), then advances every admitted request
 * by one output interval in shared launches, and retires those that reached T.  Not thread
 * safe per server.                                                                     */
typedef struct cqg_server_pars {
  uint64_t hbm_budget_bytes;  /* slot tables + state heap on the device */
  int32_t max_trajectories;   /* slots */
  int32_t max_systems;        /* distinct systems over the server's life */
  int32_t max_averages;       /* largest n_avr of a request's system */
  int32_t reserved;
  cqg_mcwf_pars mcwf;         /* shared by every request (prng_stream per request) */
} cqg_server_pars;

typedef struct cqg_server cqg_server;
void cqg_server_pars_default(cqg_server_pars* p);
int cqg_server_create(const cqg_server_pars* p, cqg_server** out);
/* Queues a request; psi0 is copied.  The request id identifies it in the calls below. */
int cqg_server_submit(cqg_server* s, const cqg_system* sys, const cqg_complex* psi0, int64_t n_traj, double T,
                      double Dt, uint64_t prng_stream, int64_t* request_id);
/* One scheduling round (admit, advance one interval, retire); returns after the round's
 * device work.  n_active / n_waiting (may be NULL): requests on the device / still queued. */
int cqg_server_round(cqg_server* s, int32_t* n_active, int32_t* n_waiting);
/* Ids of finished requests not yet collected (all of them in *n; the first cap in ids). */
int cqg_server_completed(cqg_server* s, int64_t* ids, int32_t cap, int32_t* n);
/* Result of a finished request: n_rows x n_cols sums (rows may be NULL to query the size),
 * accepted MCWF steps, times[3] = submit, admission and completion in seconds since the
 * server's creation, and the OR of its trajectories' status words.  A call with
 * cap_rows >= n_rows delivers the result and forgets the request. */
int cqg_server_result(cqg_server* s, int64_t id, double* rows, int32_t cap_rows, int32_t* n_rows, int32_t* n_cols,
                      uint64_t* steps, double* times, uint32_t* status);
/* Accepted steps of the finished requests, device time of the rounds' MCWF launches, rounds. */
int cqg_server_stats(const cqg_server* s, uint64_t* steps, double* kernel_ms, int64_t* rounds);
int cqg_server_destroy(cqg_server* s);

/* Measured FMA throughput of the current device (TFLOP/s, 2 flops per FMA) for
 * FP64 and FP32 CUDA cores: the denominator of the kernels' roofline and an
 * input of the launch-shape tuner.  Runs two short probe kernels. */
int cqg_probe_fma_peaks(double* fp64_tflops, double* fp32_tflops);

int cqg_ensemble_destroy(cqg_ensemble* ens);

/* ---- allocation-free averages ---------------------------------------------
 * No counterpart in the reference.  Sums over n_states caller-owned device states
 * (psi: n_states x D complex128, C-order, state after state) of the system's linear
 * averages: sums[c] = sum_i Re/Im <psi_i|O|psi_i>, the columns of cqg_ensemble_run
 * without the dtDid column.  For callers that cannot allocate device memory — their
 * memory belongs to another allocator (a framework pool, a serving runtime that
 * reserved the GPU up front) or they run where cudaMalloc is not allowed or would
 * synchronise the device.  Allocates nothing: the per-state intermediate sums live in
 * one fixed device array of 2^18 doubles held by every GPU that loads the library, so
 * n_states * n_avr must not exceed 262144 (larger requests fail with CQG_E_INVALID).
 * The states are used as given: they are not renormalised, and for systems with an
 * interaction picture they must already be in the frame of the output time (t0 = t, as
 * the ensemble path has them at its output times).  psi (16-byte aligned) and sums
 * (8-byte aligned) are device pointers; misaligned pointers fail with CQG_E_INVALID
 * before any work is queued.  Work is queued on `stream` (a cudaStream_t, NULL for the
 * default stream) and the call returns without waiting.  The first call on a device
 * looks up the array's device address and the device's SM count, so make that first call
 * before any stream capture, and do not use the library across a cudaDeviceReset.  All
 * calls share the array: calls whose work overlaps on the GPU race and give wrong sums.
 * The current device must be the system's device. */
int cqg_system_averages_noalloc(const cqg_system* sys, const cqg_complex* psi, int64_t n_states, double* sums,
                                void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CQG_H_INCLUDED */
