/*
 * fpsg.h — C ABI of the B200 fTWA / time-dependent Hartree-Fock trajectory engine.
 *
 * The library (libfpsg.so) replaces the trajectory loop inside FermiPhaseSpace's
 * solvers. One call of fpsg_run does what these reference functions do together:
 *
 *   FHfTWASolver::runSimulation   src/FHfTWASolver.cpp:222-556  (time loop, observables)
 *   FHfTWASolver::step_RK4_38     src/FHfTWASolver.cpp:629-661  (3/8-rule RK4 step)
 *   FHfTWASolver::derivative      src/FHfTWASolver.cpp:568-600  (d rho/dt = -i[rho, Delta])
 *   FHHFSolver::runSimulation     src/FHHFSolver.cpp:181-434
 *   FHHFSolver::step_RK4_38       src/FHHFSolver.cpp:527-558
 *   FHHFSolver::derivative        src/FHHFSolver.cpp:575-608
 *
 * and the trajectory sampling of FHfTWASolver::runSimulation (src/FHfTWASolver.cpp:342-362)
 * is fpsg_sample.  The matrices the reference solvers bind by const reference in
 * their constructors (src/FHfTWASolver.cpp:4-16: tM, U, V, extPot) are handed over
 * once with fpsg_set_system.
 *
 * Conventions
 *   - every function returns FPSG_OK (0) or a negative FPSG_ERR_* code; no C++
 *     exception crosses this boundary; fpsg_last_error() gives a readable reason;
 *   - matrices are n x n, complex double interleaved (re, im), column-major, i.e.
 *     element (i, j) is at 2*(j*n + i) — the layout of arma::cx_dmat;
 *   - host buffers are owned by the caller; device memory is owned by the context;
 *   - one context per host thread; every call blocks until its GPU work is done.
 */
#ifndef FPSG_H
#define FPSG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fpsg_ctx fpsg_ctx;

/* status codes */
enum {
    FPSG_OK              = 0,
    FPSG_ERR_INVALID     = -1,  /* bad argument or call order                          */
    FPSG_ERR_OOM         = -2,  /* device allocation failed or the context's cap was hit */
    FPSG_ERR_CUDA        = -3,  /* a CUDA runtime call failed                          */
    FPSG_ERR_TIMEOUT     = -4,  /* a bounded device-side wait gave up                  */
    FPSG_ERR_DIVERGED    = -5,  /* a trajectory went non-finite or lost its trace      */
    FPSG_ERR_STATE       = -6,  /* call made before the data it needs was set          */
    FPSG_ERR_UNSUPPORTED = -7,  /* valid request this build cannot serve               */
    FPSG_ERR_NO_DEVICE   = -8   /* no CUDA device / driver                             */
};

/* methods (fps.cpp:155-162 "method") */
enum { FPSG_METHOD_FTWA = 0, FPSG_METHOD_HF = 1 };

/* arithmetic of the RK stages */
enum {
    FPSG_PREC_FP64 = 0,          /* plain FP64, bit-identical to the FP64 oracle            */
    FPSG_PREC_FP32 = 1,          /* FP32 stages, FP64 ensemble reduction; on the resident
                                    path the state update is compensated (each element kept
                                    as FP32 plus a bf16 residual of its last update, stored
                                    back to the FP64 state at the end of a launch)           */
    FPSG_PREC_SPLIT_BF16X3 = 2,  /* dense tensor-core commutator, three-term bf16 split      */
    FPSG_PREC_SPLIT_TF32X3 = 3   /* dense tensor-core commutator, three-term tf32 split      */
};

/* Coulomb kinds (FHCoulombInteraction types, src/FHCoulombInteraction.cpp:13-76):
 * NULL -> no Hartree term; ONSITE -> U only (V ignored, src/FHfTWASolver.cpp:578);
 * DISTANCE -> U and same-spin V (plus the Fock term -rho∘V in HF). */
enum { FPSG_COULOMB_NULL = 0, FPSG_COULOMB_ONSITE = 1, FPSG_COULOMB_DISTANCE = 2 };

/* kernel selection */
enum {
    FPSG_PATH_AUTO = 0,
    FPSG_PATH_STREAM = 1,    /* one RK stage per launch, state in HBM                  */
    FPSG_PATH_RESIDENT = 2,  /* whole run per launch, state in shared memory           */
    FPSG_PATH_DENSE = 3      /* tensor-core dense commutator                           */
};

/* observables (FHSolver::setResultsToSave, src/FHSolver.cpp:34-45) */
enum {
    FPSG_OBS_DIAG     = 1u << 0,  /* Niiu, Niid           "diagDMatrix"    */
    FPSG_OBS_DIAG2    = 1u << 1,  /* N2iiu, N2iid         "diag2DMatrix"   */
    FPSG_OBS_DOUBLONS = 1u << 2,  /* NuNd                 "onSiteDoublons" */
    FPSG_OBS_WHOLE    = 1u << 3,  /* Nu, Nd (whole)       "wholeDMatrix"   */
    FPSG_OBS_ENERGIES = 1u << 4   /* E rows tH,U,V,pe,tot "energies"       */
};

/* Caller-owned host result buffers; any pointer may be NULL to skip it.
 * Site arrays are [site][time] (n x n_snapshots, row = site), matching how the
 * reference writes Niiu.row(iSite) (src/FHSolver.cpp:200-214). Values are the
 * reference's normalised observables (src/FHfTWASolver.cpp:489-551 for fTWA,
 * src/FHHFSolver.cpp:404-419 for HF), real parts. */
typedef struct fpsg_outputs {
    double* time;      /* [n_snapshots]            t*dt                                */
    double* niiu;      /* [n][n_snapshots]                                             */
    double* niid;
    double* n2iiu;
    double* n2iid;
    double* nund;
    double* energies;  /* [5][n_snapshots]  rows tH, U, V, pe, tot (src/FHSolver.cpp:276-282) */
    double* whole_u;   /* [n_snapshots][n][n] complex interleaved, ensemble-mean N (not rho) */
    double* whole_d;
    /* filled by the library */
    double  device_ms;        /* GPU time of the trajectory kernels (CUDA events)      */
    double  total_ms;         /* wall time of the call                                  */
    int64_t traj_steps;       /* trajectories x RK4 steps integrated                    */
    int64_t kernel_launches;  /* launches of this library's kernels during the call     */
    int     path_used;        /* FPSG_PATH_*                                            */
    int     reserved;
} fpsg_outputs;

/* Context flags (fpsg_create).  FPSG_FLAG_TEST_EXPIRE_WAIT is a test hook for the
 * bounded device-side waits: in every call on the dense tensor-core path, the
 * first stage launch has one thread wait on a barrier nothing arrives at, with a
 * short poll limit, before that launch allocates tensor memory or issues a copy;
 * the wait runs out, the launch returns, and the call reports FPSG_ERR_TIMEOUT
 * (its state is then not a valid integration).  No counterpart in the reference. */
#define FPSG_FLAG_TEST_EXPIRE_WAIT 0x1ull
/* FPSG_FLAG_FP32_PLAIN_STATE: FPSG_PREC_FP32 on the resident path without the
 * compensated state update (see FPSG_PREC_FP32), the plain FP32 rounding of every
 * update; a few percent faster, less accurate over long windows. */
#define FPSG_FLAG_FP32_PLAIN_STATE 0x2ull

/* Creates a context on CUDA device `device`. flags: 0, or FPSG_FLAG_* above.
 * Replaces the FHSolver constructor's binding to an FHSystem (src/FHSolver.cpp:5-9). */
int  fpsg_create(fpsg_ctx** out, int device, uint64_t flags);
void fpsg_destroy(fpsg_ctx* ctx);
const char* fpsg_last_error(const fpsg_ctx* ctx);

/* Caps the context's device memory (bytes; 0 = no cap). Allocations beyond it
 * fail with FPSG_ERR_OOM — the host-side way to exercise the out-of-memory path. */
int  fpsg_set_memory_cap(fpsg_ctx* ctx, uint64_t bytes);

/* Hamiltonian inputs. tM, U, V, extpot: n x n complex col-major (extpot/V may be
 * NULL = zero). Replaces the const references of src/FHfTWASolver.cpp:4-16 /
 * src/FHHFSolver.cpp:4-11 and the Coulomb/ext-pot switches of
 * src/FHfTWASolver.cpp:574-596. extpot_is_null mirrors
 * FHSystem::isExternalPotentialNull (it gates the potential energy row).
 * All matrices must be real symmetric (imaginary parts 0): the hot path relies on it.
 * extpot may have off-diagonal entries: like the reference, the engine adds the whole
 * matrix to Delta, and its energy row pe sums extpot_ij N_ij over every element. */
int  fpsg_set_system(fpsg_ctx* ctx, int n, const double* tM, const double* U,
                     const double* V, const double* extpot, int coulomb_kind,
                     int extpot_is_null);

/* Time-dependent site potential (a new model with no reachable counterpart in the
 * reference; FHExternalPotentialPulse, src/FHExternalPotentialPulse.cpp:86-110,
 * is the closest): v_i(t) = amp[bin(t)] * exp(-((t-t0)/td)^2/2) * proj[i], with
 * bin(t) = clamp(floor(t / bin_width), 0, n_bins-1). Added to the diagonal of Delta.
 * n_bins = 0 removes the pulse. */
int  fpsg_set_pulse(fpsg_ctx* ctx, int n_bins, const double* amp, double bin_width,
                    double t0, double td, const double* proj);

/* Injects initial samples: rho0 is [B][2][n][n] complex col-major (spin up, spin
 * down). For fTWA these are the shifted matrices rho = N - 1/2 I the reference
 * integrates (src/FHfTWASolver.cpp:358-362); for HF they are N itself. Only the
 * upper triangle and the real diagonal are read: the engine keeps the state
 * Hermitian by construction. */
int  fpsg_set_initial_samples(fpsg_ctx* ctx, int B, const double* rho0);

/* Draws B fTWA initial samples on the GPU (src/FHfTWASolver.cpp:187-198, 342-362):
 * rho_s = R_s (diag(occ_s - 1/2) + W_s∘sigma_s) R_s^H with
 * sigma_ij = sqrt((n_i + n_j - 2 n_i n_j)/2) (i != j), W_up Hermitian from the upper
 * triangle and W_down from the lower triangle of one complex Gaussian matrix W with
 * E|W_ij|^2 = 1 per trajectory (Philox4x32-10 keyed by seed, counter by trajectory
 * and element). rot_up / rot_dn: n x n complex col-major or NULL (identity). */
int  fpsg_sample(fpsg_ctx* ctx, int B, uint64_t seed, const double* occ_up,
                 const double* occ_dn, const double* rot_up, const double* rot_dn);

/* fpsg_sample for trajectories first .. first+B-1 of the seed's ensemble: a rank
 * holding a contiguous shard draws exactly the samples a single context drawing
 * them all would hold at those indices (replaces the per-node trajectory ranges
 * and per-trajectory random seeds of src/FHfTWAMPISolver.cpp:89-100, 163-171). */
int  fpsg_sample_range(fpsg_ctx* ctx, int64_t first, int B, uint64_t seed, const double* occ_up,
                       const double* occ_dn, const double* rot_up, const double* rot_dn);

/* Runs the trajectories: n_snapshots = floor(t_max/dt + 1) (src/FHSolver.cpp:100),
 * RK4 step h = dt / steps_per_snapshot. fTWA records each snapshot then steps
 * (so it also steps after the last one, src/FHfTWASolver.cpp:366-426); HF records
 * t = 0 then steps and records (src/FHHFSolver.cpp:306-401). */
int  fpsg_run(fpsg_ctx* ctx, int method, int precision, int path, double dt,
              int steps_per_snapshot, int n_snapshots, uint32_t obs_mask,
              fpsg_outputs* out);

/* Advances the state by n_steps RK4 steps from time t_start with no observables
 * (the unit the benchmark times). device_ms / launches are optional outputs. */
int  fpsg_advance(fpsg_ctx* ctx, int method, int precision, int path, double dt,
                  int steps_per_snapshot, double t_start, int n_steps,
                  double* device_ms, int64_t* launches);

/* Gradient of the time-integrated doublon occupancy,
 *     L = sum_t w_t (1/n) sum_i <n_i,up n_i,dn>(t_t),   t = 0 .. n_snapshots-1,
 * (trapezoid weights w: dt/2 at both ends, dt inside) over the fTWA trajectories
 * of the current samples, with respect to a global scale of the Coulomb matrices
 * (U, and V when present), a global scale of tM, and the pulse amplitudes of
 * fpsg_set_pulse.  Discrete adjoint of the 3/8-rule RK4 steps (the same stage
 * times as fpsg_run), checkpointing the state every `checkpoint_every` steps and
 * recomputing each segment once.  No counterpart in the reference, which has no
 * gradients.  dL_dpulse has n_bins entries; any output may be NULL.  The context
 * state is left unchanged.  device_ms: whole call; forward_ms: its first
 * (loss-only) forward pass, for the gradient / forward cost ratio.  A static
 * potential with off-diagonal entries is refused with FPSG_ERR_UNSUPPORTED (the
 * tM-scale term assumes Delta equals tM off its diagonal). */
int  fpsg_grad(fpsg_ctx* ctx, int precision, double dt, int steps_per_snapshot, int n_snapshots,
               int checkpoint_every, double* loss, double* dL_dUscale, double* dL_dtscale,
               double* dL_dpulse, double* device_ms, double* forward_ms);

/* Device memory fpsg_grad may spend on keeping the stage inputs of the last
 * checkpoint segments from its forward pass, so that the backward pass need not
 * recompute those segments (a trade of memory for time; the gradient is the same
 * to the bit either way).  bytes < 0: automatic (default), three quarters of the
 * device memory free at the call, within the memory cap; 0: recompute every
 * segment; > 0: at most that many bytes.  When every segment of the whole
 * ensemble does not fit, fpsg_grad runs the trajectories in chunks (at least one
 * trajectory per SM each, a multiple of the SM count), each a forward and a
 * reverse sweep of its own, so that every segment of a chunk is kept; the
 * gradients are the same to the bit, the loss to rounding (its ensemble sums are
 * taken in another order).  The buffer stays in the context's pool for the next
 * fpsg_grad call (memory filled before is much faster to write than a fresh
 * allocation); fpsg_set_memory_cap or fpsg_destroy releases it.  No counterpart in
 * the reference. */
int  fpsg_set_grad_memory(fpsg_ctx* ctx, int64_t bytes);

/* GPSR drift (FHGPSRSolver::step_Drift_RK4_38, src/FHGPSRSolver.cpp:168-206, with
 * the derivative of src/FHGPSRSolver.cpp:111-134): for B trajectories given as full
 * complex matrices rho[B][2][n][n] (spin up, spin down; column-major, interleaved
 * re/im, host memory; general, not Hermitian), the 3/8-rule RK4 drift increments
 * drift[B][2][n][n] over one step d_t, with Delta_up = tM + diagmat(U diag(rho_dn))
 * + extPot (no 1/2 shift, no V term; the diagonal is complex) from fpsg_set_system.
 * FP64, bit-identical to the oracle's restatement.  The caller adds the diffusion
 * part and the drift to rho, as FHGPSRSolver::step does (src/FHGPSRSolver.cpp:632-661).
 * t is the step's start time; only a time-dependent potential would use it, and a
 * pulse set with fpsg_set_pulse is refused (FPSG_ERR_UNSUPPORTED). */
int  fpsg_gpsr_drift(fpsg_ctx* ctx, int B, const double* rho, double t, double d_t, double* drift);

/* What the last successful fpsg_grad call chose: trajectories per chunk, chunks,
 * checkpoint segments, and how many of them each chunk kept from its forward
 * sweep (the others were recomputed in the reverse sweep). */
typedef struct fpsg_grad_info {
    int chunk_traj;
    int chunks;
    int segments;
    int kept_segments;
} fpsg_grad_info;
int  fpsg_last_grad_info(const fpsg_ctx* ctx, fpsg_grad_info* info);

/* One system of a batch (fpsg_run_batch): the matrices of fpsg_set_system and
 * the product-state occupations of fpsg_sample (rotation identity), drawn from
 * `seed`.  `out` receives the system's observables as fpsg_run would. */
typedef struct fpsg_system_desc {
    int n;
    const double* tM;
    const double* U;
    const double* V;
    const double* extpot;
    int coulomb_kind;
    int extpot_is_null;
    int n_traj;
    uint64_t seed;
    const double* occ_up;
    const double* occ_dn;
    fpsg_outputs* out;
} fpsg_system_desc;

/* What fpsg_run_batch chose and measured. */
typedef struct fpsg_batch_info {
    int block_threads;         /* threads per CTA picked by the autotuner             */
    int schedule;              /* 0: work items by cost, descending; 1: interleaved   */
    int grid;                  /* persistent CTAs                                     */
    int graph_nodes;           /* kernels in the captured snapshot-interval graph     */
    double tune_ms;            /* autotuning time (0 when the choice was cached)      */
    double device_ms;          /* GPU time of the integration (graph replays)         */
    int64_t traj_steps;        /* trajectories x RK4 steps over all systems           */
    int64_t kernel_launches;   /* kernel executions during the integration            */
} fpsg_batch_info;

/* Integrates several systems of different size together (no counterpart in the
 * reference, which runs one system per process): every RK stage of every
 * trajectory of every system is one persistent launch over a cost-ordered work
 * list; one snapshot interval (stages, records, per-system reductions) is
 * captured once as a CUDA graph and replayed n_snapshots times.  The block size
 * and the work order are picked by timing the candidates on the first call for
 * a batch shape (cached in the context).  precision: FP64 or FP32.  The
 * context's own system and samples are not touched.  info may be NULL. */
int  fpsg_run_batch(fpsg_ctx* ctx, const fpsg_system_desc* systems, int n_systems, int method,
                    int precision, double dt, int steps_per_snapshot, int n_snapshots,
                    uint32_t obs_mask, fpsg_batch_info* info);

/* Copies the current state out: [B][2][n][n] complex col-major (full matrices). */
int  fpsg_get_state(fpsg_ctx* ctx, double* rho);
int  fpsg_num_trajectories(const fpsg_ctx* ctx);

/* Library build information, e.g. "fpsg 0.1 sm_100a". */
const char* fpsg_version(void);

/* Ensemble sums without device allocation.  No counterpart in the reference:
 * it serves callers that cannot call cudaMalloc (work recorded into a CUDA graph,
 * hosts whose device memory belongs to another runtime's allocator, integrators
 * that keep their own trajectories).  rho: device pointer, [B][2][n][n] complex
 * interleaved col-major states (as fpsg_get_state returns them); sums: device
 * pointer to 5n doubles, receiving sum_b Re rho_up_ii, sum_b Re rho_dn_ii, their
 * squares and sum_b Re rho_up_ii * Re rho_dn_ii.  Order: chunks of 64
 * trajectories summed in ascending order, chunk partials combined in chunk order
 * with Kahan compensation — the reduction of fpsg_run's stream path, so the sums
 * equal that path's bit for bit (its resident path agrees to rounding).
 * stream: a cudaStream_t or NULL.  The call works on the calling thread's current
 * device; rho, sums and the stream must belong to it.  Allocates nothing: its
 * partial sums live in a static device array of FPSG_NOALLOC_SCRATCH_DOUBLES
 * doubles that every GPU loading the library keeps until exit; requests needing
 * more than 5 n ceil(B/64) <= FPSG_NOALLOC_SCRATCH_DOUBLES partials return
 * FPSG_ERR_INVALID (n = 100: B <= 33536).  All calls share that array, so calls
 * that overlap on the GPU race.  A call made outside a stream capture looks the
 * array's device address up (and caches it); a call made during a capture uses
 * the cached address and returns FPSG_ERR_STATE when there is none, so the first
 * call on each device (and the first after a cudaDeviceReset) must come before
 * any capture.  If the calling thread already has a CUDA error pending, the call
 * returns FPSG_ERR_CUDA without launching and leaves that error pending. */
#define FPSG_NOALLOC_SCRATCH_DOUBLES 262144
int fpsg_ensemble_sums_noalloc(const double* rho, int B, int n, double* sums, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* FPSG_H */
