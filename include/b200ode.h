/* b200ode -- C ABI of the B200 batched stiff-chemistry BDF integrator.
 *
 * This is the boundary the host-side Integrator subclass (B200BDFIntegrator,
 * include/b200ode_integrator.hpp) calls.  It replaces, for one batch of
 * cells, what the reference's GPU path does inside
 *   CVodeIntegratorGPU::integrate / integrateBatch
 *     src/Integrators/CVodeIntegratorGPU.cpp:30-126
 *   (calc_gpu_points, init_memory_gpu, N_VNew_Cuda, CVodeCreate(CV_BDF),
 *    SUNMatrix_MagmaDenseBlock, SUNLinSol_MagmaDense, CVode(..., CV_NORMAL),
 *    saveGPUArrayResults; src/Integrators/Drivers/CVodeGPUDriver.cu:28-398)
 * and what the serial oracle path does per cell in
 *   CVodeIntegrator::integrateSystem  src/Integrators/CVodeIntegrator.cpp:98-155.
 *
 * Semantics are those of the serial CVODE path: every cell runs its own
 * variable-order BDF (own step size, order and error test), to tout = t1 in
 * CV_NORMAL mode, with scalar reltol/abstol (CVodeSStolerances) and
 * max_steps (CVodeSetMaxNumSteps, 10000 in the reference).  The state of a cell
 * is [T, Y_0 .. Y_{nsp-2}]; the last species is returned as 1 - sum(Y_k)
 * (CVodeIntegrator.cpp:79-96).
 *
 * Data layout: structure of arrays, cell index innermost.  Y is nsp x n_cells
 * (Y[k * n_cells + c]), T and P are n_cells long.  Plain pointers, no C++ types,
 * no exceptions cross the ABI.  The caller owns every host buffer; the library
 * owns its device buffers.  A handle is used by one host thread at a time.
 */
#ifndef B200ODE_H
#define B200ODE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct b200ode_handle b200ode_handle;

typedef enum {
    B200ODE_OK = 0,
    B200ODE_ERR_INVALID = 1,     /* bad argument (null pointer, size, tolerance ...) */
    B200ODE_ERR_MECHANISM = 2,   /* unknown mechanism or species-count mismatch */
    B200ODE_ERR_CUDA = 3,        /* CUDA runtime error (message in b200ode_last_error) */
    B200ODE_ERR_ALLOC = 4,       /* device or pinned allocation failed */
    B200ODE_ERR_NO_DEVICE = 5,   /* no usable CUDA device */
    B200ODE_ERR_BUSY = 6,        /* serving queue full */
    B200ODE_ERR_NOT_READY = 7    /* serving request still in flight */
} b200ode_status;

/* Per-cell integration status: CVODE return codes (CVode() return values). */
enum {
    B200ODE_CELL_SUCCESS = 0,
    B200ODE_CELL_TOO_MUCH_WORK = -1,   /* CV_TOO_MUCH_WORK: max_steps reached */
    B200ODE_CELL_TOO_MUCH_ACC = -2,    /* CV_TOO_MUCH_ACC */
    B200ODE_CELL_ERR_FAILURE = -3,     /* CV_ERR_FAILURE: 7 error-test failures in one step */
    B200ODE_CELL_CONV_FAILURE = -4,    /* CV_CONV_FAILURE: 10 convergence failures in one step */
    B200ODE_CELL_ILL_INPUT = -22,      /* CV_ILL_INPUT: the cell's pressure is not > 0 (cell left as given) */
    B200ODE_CELL_TOO_CLOSE = -27       /* CV_TOO_CLOSE: t1 too close to t0 */
};

typedef enum { B200ODE_FP64 = 0, B200ODE_MIXED = 1 } b200ode_precision;

/* Reactor formulation.  CONP: constant pressure (the reference's pyJac build,
 * src/Mechanism/CPU/dydt.c:7-133): P per cell is held, enthalpy conserved.
 * CONV: constant volume (pyJac's CONV branch, dydt.c:135-265, which the
 * reference ships but does not compile): the P given per cell is the initial
 * pressure, the cell's density rho = P W / (R T) of its initial state is held,
 * the pressure follows the state (P = rho R T / W) and internal energy is
 * conserved. */
typedef enum { B200ODE_CONP = 0, B200ODE_CONV = 1 } b200ode_formulation;

typedef struct {
    double reltol;            /* CVodeSStolerances reltol (reference: 1e-6) */
    double abstol;            /* CVodeSStolerances abstol (reference: 1e-10) */
    int32_t max_steps;        /* CVodeSetMaxNumSteps (reference: 10000) */
    int32_t max_order;        /* BDF max order, 1..5 (CVODE default 5) */
    int32_t precision;        /* B200ODE_FP64 or B200ODE_MIXED (FP32 Jacobian/LU/solve) */
    int32_t refine;           /* mixed only: 1 = one FP64-residual refinement sweep per solve */
    int32_t persistent;       /* 1 = persistent kernel + device work queue; 0 = one launch per BDF step */
    int32_t warps_per_block;  /* 0 = from the autotuner / occupancy */
    int32_t blocks_per_sm;    /* 0 = from occupancy, with the kernel's register variant (up to 255,
                                 168 or 128 registers a thread; 128 only below 32 unknowns) that
                                 keeps the most CTAs resident; n >= 3 x 4 / warps_per_block
                                 selects the 168-register variant, n >= 4 x 4 / warps_per_block
                                 the 128-register one where built */
    int32_t queue_chunk;      /* persistent form: consecutive cells a warp claims per work-queue
                                 access, 1..64 (0 = 1); larger chunks trade queue traffic for
                                 tail balance.  Results do not depend on it. */
    int32_t use_graph;        /* one-launch-per-step form: capture the step launches in a CUDA graph */
    int32_t device;           /* CUDA device ordinal (-1 = current) */
    int32_t profile_phases;   /* 1 = accumulate per-phase device cycles into b200ode_stats */
    int32_t formulation;      /* B200ODE_CONP (default) or B200ODE_CONV */
    int32_t cta_helpers;      /* mechanisms whose Newton matrix fills an SM (one cell per SM):
                                 1 (default) = the CTA's other three warps take shares of the
                                 cell's reaction groups and LU updates; 0 = one warp per cell.
                                 Results are the same either way. */
    /* Wait limits of that hand-off in SM clock cycles (0 = defaults: join ~2 s, drain ~2 s,
       helper idle ~10 s).  Diagnostics for the recovery paths: when warp 0's wait for a
       share (join) runs out it waits once more (drain); late shares that arrive then leave
       the cell's results unchanged and warp 0 goes on alone; if the drain runs out too,
       the CTA fails its current cell and every later cell it claims with
       B200ODE_CELL_ERR_FAILURE (later ones left as given). */
    int64_t helper_join_cycles;
    int64_t helper_drain_cycles;
    int64_t helper_idle_cycles;
    /* Largest number of cells one launch sequence takes (0 = as many as fit: 80 % of the
       free device memory over the per-cell footprint, as the reference's calc_gpu_points
       sizes its batches).  A larger call runs as consecutive launches over contiguous
       chunks of cells; results do not depend on the chunking. */
    int64_t max_cells_per_launch;
} b200ode_options;

/* Optional per-cell counters (CVodeGetNum* equivalents) and call totals.  Any
 * per-cell pointer may be NULL.  Totals and timings are always filled. */
typedef struct {
    int32_t* nst;        /* steps */
    int32_t* nfe;        /* RHS evaluations */
    int32_t* nje;        /* Jacobian evaluations */
    int32_t* nsetups;    /* Newton-matrix setups (LU factorizations) */
    int32_t* nni;        /* Newton iterations (linear solves) */
    int32_t* ncfn;       /* nonlinear convergence failures */
    int32_t* netf;       /* error-test failures */
    int64_t total_nst, total_nfe, total_nje, total_nsetups, total_nni, total_ncfn, total_netf;
    int64_t n_failed;        /* cells whose status != B200ODE_CELL_SUCCESS */
    double h2d_ms, kernel_ms, d2h_ms;   /* device-timed phases of the last call */
    int32_t gpu_launches;    /* kernels this library launched in the last call */
    int64_t phase_cycles[5]; /* profile_phases: SM cycles summed over warps in RHS, Jacobian,
                                LU, triangular solves, and the whole kernel (persistent form) */
} b200ode_stats;

/* Fill *opts with the reference's settings (1e-6 / 1e-10 / 10000 / order 5),
 * mixed precision, persistent kernel. */
void b200ode_default_options(b200ode_options* opts);

/* Create a handle for a mechanism compiled into the library: "gri30", "h2o2",
 * "nDodecane_Reitz" (".yaml" suffix optional), "h2_li_2004" or
 * "ESTiMatE-Mech_04042022" (".xml" optional).  ESTiMatE (214 species) runs in
 * B200ODE_MIXED only: its FP64 Newton matrix exceeds an SM's shared memory
 * (B200ODE_ERR_INVALID).
 * Replaces the per-batch set-up of CVodeIntegratorGPU::integrateBatch
 * (CVodeIntegratorGPU.cpp:44-100) and CVodeIntegrator::init's NSP check
 * (CVodeIntegrator.cpp:34-50).  opts may be NULL (defaults). */
b200ode_status b200ode_create(const char* mech_name, const b200ode_options* opts,
                              b200ode_handle** out);
void b200ode_destroy(b200ode_handle* h);

/* Number of species of a mechanism by name, without a device (the reference's
 * NSP, src/Mechanism/CPU/mechanism.h); -1 for an unknown name.  Lets a host
 * check a mesh against the mechanism before any GPU work. */
int32_t b200ode_mechanism_species(const char* mech_name);

/* Number of species of the handle's mechanism (the reference's NSP). */
int32_t b200ode_num_species(const b200ode_handle* h);

/* Integrate n_cells cells from t0 to t1 (host buffers, synchronous).
 * P: per-cell pressure [Pa] (n_cells) or NULL to use P_scalar (the reference's
 * IntegratorConfig::pressure, Integrator.hpp:13-19).  T (n_cells) and Y
 * (nsp x n_cells, SoA) are read and overwritten.  cell_status (n_cells) may be
 * NULL.  stats may be NULL.  Cells that fail keep the last accepted state, as
 * CVode returns it. */
b200ode_status b200ode_integrate(b200ode_handle* h, int64_t n_cells, const double* P,
                                 double P_scalar, double* T, double* Y, double t0, double t1,
                                 int32_t* cell_status, b200ode_stats* stats);

/* Same on device-resident buffers (no host copies; stream is a cudaStream_t or
 * NULL for the legacy default stream).  Asynchronous with respect to the host
 * unless stats is non-NULL (then it synchronizes the stream to fill totals;
 * per-cell counter pointers must be device pointers). */
b200ode_status b200ode_integrate_device(b200ode_handle* h, int64_t n_cells, const double* d_P,
                                        double P_scalar, double* d_T, double* d_Y, double t0,
                                        double t1, int32_t* d_cell_status, b200ode_stats* stats,
                                        void* stream);

/* Size of the static device scratch of b200ode_integrate_device_noalloc. */
#define B200ODE_NOALLOC_SCRATCH_BYTES (32u << 20)

/* b200ode_integrate_device without any device allocation.  No counterpart in
 * the reference.
 *
 * For callers that must not allocate device memory while they integrate: a flow
 * solver whose memory pool has taken the whole GPU at start-up, or one that
 * cannot accept, in the middle of its time step, the device-wide
 * synchronization of cudaFree (b200ode_integrate_device frees and re-allocates
 * its per-handle scratch when a larger launch outgrows it).  Arguments, results
 * and per-cell semantics are those of b200ode_integrate_device; the caller
 * passes every input and output buffer.  This call makes no cudaMalloc, cudaFree
 * or other allocating call: the work-queue head, the call totals and the
 * per-warp Newton scratch live in one static device array of
 * B200ODE_NOALLOC_SCRATCH_BYTES (32 MiB), which every GPU that loads this
 * library keeps until the process exits.
 *
 *  - Always runs the persistent kernel (options.persistent and use_graph are
 *    not used), with the launch shape b200ode_integrate_device would use.  A
 *    launch needs 256 bytes + resident cells x per-cell scratch (17.4 KB for
 *    GRI-Mech 3.0 in mixed precision, 28.6 KB in FP64); one that needs more than
 *    the array is refused with B200ODE_ERR_INVALID and the numbers in
 *    b200ode_last_error().  On a 148-SM B200 the default launch of every
 *    compiled-in mechanism and precision fits (the largest: the 214-species
 *    kerosene mechanism, 148 cells x 210 KB = 31.1 MB, and GRI-Mech 3.0 mixed,
 *    1,776 resident cells x 17.4 KB = 30.8 MB).  The number of cells is not
 *    limited.
 *  - The first call on a device looks up the array's device address there
 *    (and, with lazy module loading, is when the CUDA driver loads this
 *    library's kernels onto that device).  Make that first call before any
 *    stream capture.
 *  - Every call on a device shares the one array, which keeps the previous
 *    call's contents; each call clears the part that must start at zero.  Calls
 *    that overlap on the GPU (different streams, handles or host threads without
 *    ordering between them) race on the array and give wrong results.
 *  - Asynchronous unless stats is non-NULL (then it synchronizes the stream to
 *    fill the totals). */
b200ode_status b200ode_integrate_device_noalloc(b200ode_handle* h, int64_t n_cells, const double* d_P,
                                                double P_scalar, double* d_T, double* d_Y, double t0,
                                                double t1, int32_t* d_cell_status, b200ode_stats* stats,
                                                void* stream);

/* Chemistry source terms alone, one GPU warp per cell (host buffers).
 * Counterparts of the reference's batched pyJac kernels dydt_cvode_GPU /
 * kernel_dydt (src/Integrators/Drivers/CVodeGPUDriver.cu:28-65, 299-313) and of
 * pyJac's dydt (src/Mechanism/CPU/dydt.c:7): T, Y as in b200ode_integrate;
 * dTdt (n_cells) and dYdt ((nsp-1) x n_cells, SoA) receive d/dt of the state
 * [T, Y_0 .. Y_{nsp-2}].  Arithmetic in FP64. */
b200ode_status b200ode_eval_rhs(b200ode_handle* h, int64_t n_cells, const double* P, double P_scalar,
                                const double* T, const double* Y, double* dTdt, double* dYdt);

/* Analytic Jacobian, one GPU warp per cell.  Counterpart of
 * jacobian_cvode_GPU / kernel_eval_jacob (CVodeGPUDriver.cu:67-106, 338-354)
 * and pyJac's eval_jacob (src/Mechanism/CPU/jacob.c:3): jac receives, per cell,
 * nsp x nsp column-major d f_i / d y_j with y = [T, Y_0 .. Y_{nsp-2}]
 * (jac[c*nsp*nsp + i + nsp*j]).  Computed in the handle's Newton-matrix
 * precision (FP32 for B200ODE_MIXED, FP64 otherwise). */
b200ode_status b200ode_eval_jacobian(b200ode_handle* h, int64_t n_cells, const double* P,
                                     double P_scalar, const double* T, const double* Y, double* jac);

/* Mixture specific enthalpy [J/kg] of each cell from T (n_cells) and Y
 * (nsp x n_cells, SoA, all species): h = sum_k Y_k h_k(T) / W_k with the
 * mechanism's NASA-7 polynomials (host buffers; _device: device buffers, async
 * on stream).  The reference's CVODE integrators leave the Mesh's ENTHA as it
 * was; its Cantera integrator writes it after integrating
 * (src/Integrators/CanteraIntegrator.cpp:93).  This gives the CVODE-semantics
 * path an enthalpy consistent with the integrated state. */
b200ode_status b200ode_eval_enthalpy(b200ode_handle* h, int64_t n_cells, const double* T, const double* Y,
                                     double* h_mass);
b200ode_status b200ode_eval_enthalpy_device(b200ode_handle* h, int64_t n_cells, const double* d_T,
                                            const double* d_Y, double* d_h_mass, void* stream);

/* Autotuner: integrates a sample of the given cells (the first min(n_cells,
 * 192 x SMs), about 16 per resident warp, or two per SM for the 214-species
 * mechanism; device buffers as
 * b200ode_integrate_device, left unmodified) with the persistent kernel and
 * keeps the fastest choice in the handle's options, which later calls on this
 * handle use.  Stage 1 times every launch shape: 4, 2 or 1 warps (cells) per
 * CTA x the register variant that keeps the most CTAs resident or the
 * 168-register one, and for the
 * 214-species mechanism also the threads per cell (one 4-warp CTA per cell
 * with helper warps, or one warp), skipping shapes whose shared memory exceeds
 * a CTA's; stage 2 times the work-queue chunk (1, 2 or 8 cells per claim) on
 * the chosen shape.  Results do not depend on any of these choices.  The chosen
 * warps_per_block and blocks_per_sm are also returned (either pointer may be
 * NULL); b200ode_get_options returns all of them (cta_helpers, queue_chunk
 * included).  No reference counterpart: MAGMA's batched LU picks its kernel by
 * a fixed size crossover (ext/magma-2.6.2/control/get_batched_crossover.cpp). */
b200ode_status b200ode_autotune(b200ode_handle* h, int64_t n_cells, const double* d_P, double P_scalar,
                                const double* d_T, const double* d_Y, double t0, double t1,
                                int32_t* warps_per_block, int32_t* blocks_per_sm);

/* The options a handle uses now (after creation defaults were resolved and any
 * autotuning).  No reference counterpart. */
b200ode_status b200ode_get_options(const b200ode_handle* h, b200ode_options* out);

/* Diagnostic: measured FP64 FMA throughput of a device (GFLOP/s), the
 * denominator of the FP64-pipe roofline this library reports.  No reference
 * counterpart (a measurement helper). */
b200ode_status b200ode_fp64_peak(int32_t device, double* gflops);

/* Diagnostic: measured FP32 FMA throughput of a device (GFLOP/s), the
 * denominator of the FP32 part of the roofline (the mixed form's Newton matrix,
 * LU and solves).  No reference counterpart (a measurement helper). */
b200ode_status b200ode_fp32_peak(int32_t device, double* gflops);

/* ------------------------------------------------------------------ serving
 * A request loop for an operator-split flow solver that sends chemistry batches
 * (different sizes, different mechanisms) every flow step.  No counterpart in the
 * reference, whose integrators are synchronous (Integrator::integrate,
 * Integrator.hpp:22-40); the per-request work is exactly b200ode_integrate's.
 *
 * Continuous batching: a host thread admits queued requests as soon as a
 * stream slot is free and the request's device footprint fits in what is free
 * of the server's device budget (reserved once at creation; admission is
 * bookkeeping, no cudaMalloc while kernels run).  Admitted requests run on
 * their own streams, so their kernels overlap on the GPU: thread blocks of a
 * later request take SMs as those of earlier requests finish.  Admission is
 * first-in first-out; a request that does not fit lets smaller later ones pass
 * at most 8 times before the queue waits for it.  Each cell's result does not
 * depend on what else is in flight. */
typedef struct b200ode_server b200ode_server;

typedef struct {
    b200ode_options solver;     /* tolerances, precision, launch shape of every request */
    int64_t hbm_budget_bytes;   /* device bytes requests in flight may hold (0 = 25 % of free memory) */
    int32_t max_inflight;       /* requests on the GPU at once = streams (0 = 4) */
    int32_t max_queued;         /* requests waiting for admission before submit returns BUSY (0 = 4096) */
    int32_t chunk_cells;        /* a request runs as consecutive launches of at most this many cells,
                                   each launched when the previous one is done, so other requests'
                                   blocks take SMs in between; its device footprint is one chunk's
                                   (0 = 32768) */
} b200ode_server_options;

typedef struct {
    int64_t n_cells;
    int64_t n_failed;          /* cells whose status != B200ODE_CELL_SUCCESS */
    int64_t total_nst, total_nni;
    int64_t footprint_bytes;   /* device bytes the request held while in flight (one chunk's) */
    double queue_ms;           /* submit -> admitted */
    double device_ms;          /* first chunk's H2D to last chunk's D2H on its stream (CUDA
                                  events; includes the host gaps between chunks) */
    double latency_ms;         /* submit -> results in the caller's buffers */
} b200ode_request_info;

typedef struct {
    int64_t submitted, completed, failed_requests, cells_completed;
    double p50_latency_ms, p99_latency_ms, max_latency_ms, mean_queue_ms;
    double cells_per_sec;          /* completed cells / (last completion - first submit) */
    int32_t max_concurrent;        /* most requests in flight at once */
    int64_t budget_bytes, peak_bytes;
} b200ode_server_report;

void b200ode_default_server_options(b200ode_server_options* opts);
b200ode_status b200ode_server_create(const b200ode_server_options* opts, b200ode_server** out);
/* Waits for requests in flight; requests still queued are dropped. */
void b200ode_server_destroy(b200ode_server* s);

/* Queue one batch: arguments as b200ode_integrate (host buffers).  T, Y and
 * cell_status (may be NULL) receive the results; P, T, Y and cell_status must
 * stay valid and untouched until b200ode_poll reports the request done.
 * Returns B200ODE_ERR_BUSY when max_queued requests wait, B200ODE_ERR_INVALID
 * when one chunk of the request alone exceeds the server's device budget. */
b200ode_status b200ode_submit(b200ode_server* s, const char* mech_name, int64_t n_cells, const double* P,
                              double P_scalar, double* T, double* Y, double t0, double t1,
                              int32_t* cell_status, uint64_t* request_id);

/* B200ODE_OK when the request is done (results in the caller's buffers, info
 * filled if non-NULL, the id retired); B200ODE_ERR_NOT_READY if it is still
 * queued or running after waiting up to wait_ms (0 = do not wait, -1 = until
 * done); another status if the request failed (message in b200ode_last_error). */
b200ode_status b200ode_poll(b200ode_server* s, uint64_t request_id, int32_t wait_ms,
                            b200ode_request_info* info);

/* Latency percentiles and throughput over the requests completed so far. */
b200ode_status b200ode_server_get_report(b200ode_server* s, b200ode_server_report* report);

/* Message of the last error on this thread ("" if none). */
const char* b200ode_last_error(void);

/* Library version string. */
const char* b200ode_version(void);

#ifdef __cplusplus
}
#endif
#endif /* B200ODE_H */
