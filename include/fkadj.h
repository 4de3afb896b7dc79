/*
 * fkadj.h -- C ABI of libfkadj, a B200 (sm_100a) Fenton-Karma forward /
 * adjoint engine.  Plain pointers and sizes only; every entry point returns
 * an fkadj_status and never exits the process.
 *
 * It is the drop-in seam behind the reference's two MEX gateways
 * (agarzon27/adjoint-optimization):
 *   fkadj_forward  replaces  fk_forward_Et_comp
 *                  (decl src/cuda/fk_forward_Et_param_mex.cpp:27-29,
 *                   def  src/cuda/fk_forward_Et_mono_PARAMETERS.cu:646-849)
 *   fkadj_grad     replaces  fk_grad_Et_comp
 *                  (decl src/cuda/fk_grad_Et_param_mex.cpp:3-6,
 *                   def  src/cuda/fk_grad_Et_mono_PARAMETERS.cu:1569-1938)
 * with the same argument meaning and layouts:
 *   Et[nt+1]          E sample i at t = i*dt
 *   y_ini[3*n_num]    compact active cells in increasing linear index, [u;v;w]
 *   active_index[n]   n = nrows*ncols, linear index k = i*ncols + j,
 *                     1-based compact index, 0 = hole
 *   gh_num[n_num]     ghost_lr (-1/0/+1 for the shipped grids); the source is
 *                     E(t) * (Du*2/h) * gh_num on u
 *   S                 n_num x n_num objective matrix in CSC (Jc, Ir, Sv)
 *   ys[ns][3n], yf[3n] dense grids with NaN at holes
 * Differences (all additive): the FK parameter set is a runtime argument
 * (the reference compiles it in, src/cuda/fk_parameters_00_05_alpha_0p8_dx_0p035.h),
 * the CSC matrix replaces the mxArray, and an optional options struct selects
 * the gradient mode, the trajectory checkpoint policy and the CUDA stream.
 * The reference's param_str output is returned by fkadj_param_string.
 */
#ifndef FKADJ_H
#define FKADJ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FKADJ_ABI_VERSION 1

typedef enum {
    FKADJ_OK = 0,
    FKADJ_ERR_ARG = 1,        /* invalid argument (sizes, null pointers, mismatch) */
    FKADJ_ERR_CUDA = 2,       /* a CUDA runtime call failed; see fkadj_last_error */
    FKADJ_ERR_NOMEM = 3,      /* device or host allocation failed */
    FKADJ_ERR_NUMERIC = 4,    /* non-finite value in an active cell */
    FKADJ_ERR_NODEVICE = 5,   /* no CUDA device / kernels not loadable */
    FKADJ_ERR_BUSY = 6,       /* serving queue full */
    FKADJ_ERR_TIMEOUT = 7     /* bounded wait expired */
} fkadj_status;

/* FK constants, diffusivities and spacing h (cm).  Field order and meaning
 * of src/cuda/fk_parameters_00_05_alpha_0p8_dx_0p035.h:2-23. */
typedef struct {
    double u_c, u_v, tau_d, tau_v1_minus, tau_v2_minus, tau_v_plus, tau_0, tau_r,
           tau_si, u_csi, k_fk, tau_w_minus, tau_w_plus, Du, Dv, Dw, ksm, h;
} fkadj_params;

typedef enum {
    FKADJ_GRAD_REF = 0,   /* the reference's continuous adjoint: Hermite midpoint
                             states, backward RK4 on -dz/dt = (L+J_F)^T z;
                             gradE[i] = alpha*Et[i] - z(t_i).gh  (cu-G:1924-1926) */
    FKADJ_GRAD_EXACT = 1  /* discrete adjoint of the RK4 sweep and of the
                             not-a-knot spline; gradE[i] = (1/dt) dLcost/dEt[i] */
} fkadj_grad_mode;

typedef enum {
    FKADJ_CKPT_AUTO = 0,     /* FULL when it fits the budget, else whichever of SQRT and
                                BINOMIAL fits and recomputes fewer forward steps */
    FKADJ_CKPT_FULL = 1,     /* every state resident on the device */
    FKADJ_CKPT_SQRT = 2,     /* ~sqrt(nt) checkpoints, segments recomputed backward */
    FKADJ_CKPT_BINOMIAL = 3  /* binomial (revolve) schedule within ckpt_budget_bytes */
} fkadj_ckpt_policy;

typedef struct {
    int grad_mode;              /* fkadj_grad_mode (default FKADJ_GRAD_REF) */
    int ckpt_policy;            /* fkadj_ckpt_policy (default AUTO) */
    int64_t ckpt_budget_bytes;  /* device bytes for stored states; 0 = 60% of free */
    int device;                 /* CUDA device ordinal; -1 = current */
    void *stream;               /* cudaStream_t to run on; NULL = library stream */
    int tile;                   /* kernel tile preset (0 = autotuned default) */
    int verbose;                /* 0 = silent */
} fkadj_options;

/* Fills *opt with the defaults. */
void fkadj_default_options(fkadj_options *opt);
/* The reference's default FK parameter set (the header above) with h = dx. */
void fkadj_default_params(fkadj_params *p, double dx);

/* Forward sweep (replaces fk_forward_Et_comp, cu-F:646-849).  Writes state
 * snapshots every nstep steps into ys (ns of them, the final step excluded when
 * nt/nstep is an integer, as compute_ns does in fk_forward_Et_param_mex.cpp:7-25)
 * and the final state into yf.  ys may be NULL when ns == 0. */
fkadj_status fkadj_forward(const fkadj_params *p, double dt, const double *Et, int nt,
                           const double *y_ini, const int *active_index, int nrows,
                           int ncols, int n_num, const double *gh_num, int nstep, int ns,
                           double *ys, double *yf, const fkadj_options *opt);

/* Objective and gradient (replaces fk_grad_Et_comp, cu-G:1569-1938):
 * L0 = sum_v gamma[v] y_v(T)^T S y_v(T), LE = dt*sum Et^2,
 * Lcost = L0/2 + alpha*LE/2, gradE[nt+1].  yf (may be NULL) receives the
 * final forward state (dense NaN grid). */
fkadj_status fkadj_grad(const fkadj_params *p, double dt, const double *Et, int nt,
                        const double *y_ini, const int *active_index, int nrows, int ncols,
                        int n_num, const double *gh_num, const double *gamma,
                        int64_t S_ncol, const int64_t *S_colptr, const int64_t *S_rowidx,
                        const double *S_val, double alpha, double *L0, double *LE,
                        double *Lcost, double *gradE, double *yf, const fkadj_options *opt);

/* fkadj_forward and fkadj_grad build their problem afresh on every call.  They
 * keep its device memory (a stream-ordered pool per device) and its pinned
 * host staging for the next call: freeing them at the end of each call, as
 * the reference's MEX call does, was measured to stall a call by up to 0.8 s
 * at times.  That memory stays with the process; this hands it back to the
 * devices and the host (no counterpart in the reference).
 * FKADJ_ONESHOT_POOL=0 in the environment allocates device memory per call. */
fkadj_status fkadj_release_cached_memory(void);

/* Parameter provenance text (the role of the reference's param_str).  The
 * returned string is owned by the library and valid until the next call from
 * the same thread. */
const char *fkadj_param_string(const fkadj_params *p);

/* Message of the last failure on this thread ("" if none). */
const char *fkadj_last_error(void);

/* ------------------------------------------------------------------------
 * Resident problems: geometry, objective and work buffers stay on the device
 * between calls (optimisation loops, line-search probes, serving).
 * --------------------------------------------------------------------- */
typedef struct fkadj_problem fkadj_problem;

fkadj_status fkadj_problem_create(fkadj_problem **out, const fkadj_params *p, double dt, int nt,
                                  const int *active_index, int nrows, int ncols, int n_num,
                                  const double *gh_num, const double *gamma, int64_t S_ncol,
                                  const int64_t *S_colptr, const int64_t *S_rowidx,
                                  const double *S_val, double alpha, const fkadj_options *opt);
void fkadj_problem_destroy(fkadj_problem *pb);

/* Device bytes the problem holds (geometry + work + trajectory store). */
int64_t fkadj_problem_device_bytes(const fkadj_problem *pb);

/* Objective only (forward sweep, no trajectory storage). */
fkadj_status fkadj_problem_objective(fkadj_problem *pb, const double *Et, const double *y_ini,
                                     double *L0, double *LE, double *Lcost, double *yf);

/* Objective + gradient through the problem's buffers.  In both calls y_ini
 * may be NULL to re-use the initial state of the previous call, which stays
 * resident on the device. */
fkadj_status fkadj_problem_grad(fkadj_problem *pb, const double *Et, const double *y_ini,
                                double *L0, double *LE, double *Lcost, double *gradE,
                                double *yf);

/* Timing of the last call on the problem, milliseconds of device time:
 * out[0] forward, out[1] backward (incl. recompute), out[2] total. */
void fkadj_problem_last_timing(const fkadj_problem *pb, double out[3]);

/* Number of kernel launches the last call on the problem issued. */
int64_t fkadj_problem_last_launches(const fkadj_problem *pb);

/* Trajectory store of the last gradient on the problem (no counterpart in the
 * reference, which keeps every state in host memory, cu-G:1658-1664):
 * out[0] policy (fkadj_ckpt_policy FULL/SQRT/BINOMIAL; 0 before the first
 * gradient), out[1] stored state slots, out[2] segment / scratch slots,
 * out[3] forward steps the backward sweep recomputes. */
void fkadj_problem_last_plan(const fkadj_problem *pb, int64_t out[4]);

/* How the reference-mode backward step runs (no counterpart in the reference,
 * which launches seven kernels per step, cu-G:1874-1895): out[0] 0 = midpoint
 * and step kernels, 1 = one fused kernel reading the cached J_F(y)^T, 2 = one
 * fused kernel evaluating it; out[1..3] the fused kernel's tile (TX, TY,
 * threads), 0 for the split kernels (fkadj_problem_tiles has theirs).  The
 * split kernels run unless FKADJ_ADJ_PATH (fused, fused-recompute) selects the
 * fused kernel, whose preset the autotuner then times at the first gradient. */
void fkadj_problem_adjoint_kernel(const fkadj_problem *pb, int out[4]);

/* Sampled per-kernel device time: when enabled, CUDA events bracket about one
 * in (nt/100) launches of each kernel kind during the following calls.
 * kernel: 0 forward step, 1 adjoint midpoint, 2 adjoint step.  Reports the
 * average milliseconds per launch of the last call and the sample count.
 * No reference counterpart (the reference has no timers besides tic/toc in
 * src/cuda/simple_grad_desc.m:80-86). */
void fkadj_problem_set_profiling(fkadj_problem *pb, int enable);
/* Tile presets in use (autotuned or fixed) for the forward step, adjoint
 * midpoint, adjoint step and exact adjoint step: out[k] = preset index, with
 * (tx, ty, threads) of each preset in shapes[3k..3k+2] when shapes != NULL. */
void fkadj_problem_tiles(const fkadj_problem *pb, int out[4], int shapes[12]);
void fkadj_problem_kernel_time(const fkadj_problem *pb, int kernel, double *avg_ms, int64_t *samples);

/* ------------------------------------------------------------------------
 * Batches: many independent problems (different grids, horizons, pulses,
 * obstacle layouts) advanced together.  Every tick takes the next step of
 * every running job and runs them as at most three launches of persistent
 * kernels over a work queue of (problem, tile) items.  No reference
 * counterpart (the reference runs one instance per MATLAB call,
 * src/cuda/simple_grad_desc.m:82).  Problems of a batch live on the batch's
 * stream; one job per problem runs at a time; at most 128 jobs run at once.
 * --------------------------------------------------------------------- */
typedef struct fkadj_batch fkadj_batch;

fkadj_status fkadj_batch_create(fkadj_batch **out, const fkadj_options *opt);
void fkadj_batch_destroy(fkadj_batch *b);
/* Adds a resident problem (geometry, objective); grad_mode / ckpt_policy /
 * ckpt_budget_bytes as in fkadj_options.  S may be NULL for forward-only. */
fkadj_status fkadj_batch_add_problem(fkadj_batch *b, const fkadj_params *p, double dt, int nt,
                                     const int *active_index, int nrows, int ncols, int n_num,
                                     const double *gh_num, const double *gamma, int64_t S_ncol,
                                     const int64_t *S_colptr, const int64_t *S_rowidx, const double *S_val,
                                     double alpha, int grad_mode, int ckpt_policy, int64_t ckpt_budget_bytes,
                                     int *problem_id);
fkadj_status fkadj_batch_remove_problem(fkadj_batch *b, int problem_id);
/* Queues an objective (want_grad = 0) or objective + gradient job; y_ini may be
 * NULL to re-use the problem's resident initial state. */
fkadj_status fkadj_batch_submit(fkadj_batch *b, int problem_id, const double *Et, const double *y_ini,
                                int want_grad, int *job_id);
/* One tick (*active receives the number of unfinished jobs), or ticks until
 * every job is done. */
fkadj_status fkadj_batch_tick(fkadj_batch *b, int *active);
fkadj_status fkadj_batch_run(fkadj_batch *b);
int fkadj_batch_job_done(const fkadj_batch *b, int job_id);
/* Results of a finished job: gradE receives min(n_gradE, nt+1) values. */
fkadj_status fkadj_batch_result(fkadj_batch *b, int job_id, double *L0, double *LE, double *Lcost,
                                double *gradE, int64_t n_gradE);
fkadj_status fkadj_batch_release(fkadj_batch *b, int job_id);
/* out[0] kernel launches, out[1] ticks, out[2] device bytes held. */
void fkadj_batch_stats(const fkadj_batch *b, int64_t out[3]);

/* ------------------------------------------------------------------------
 * Serving: a worker thread owns the GPU and runs a batch continuously.
 * Requests (any thread) queue in arrival order and are admitted between ticks
 * while their estimated device footprint fits hbm_budget_bytes (0 = 80% of
 * free memory) and fewer than 128 run; admitted requests share every launch
 * with the running ones and free their memory when they finish.  All waits are
 * bounded.  No reference counterpart.  options.grad_mode / ckpt_policy apply
 * to every request (ckpt_policy FULL or else sqrt checkpoints).
 * --------------------------------------------------------------------- */
typedef struct fkadj_server fkadj_server;

fkadj_status fkadj_server_create(fkadj_server **out, const fkadj_options *opt, int64_t hbm_budget_bytes);
/* Finishes the queued and running requests, then stops the worker. */
void fkadj_server_destroy(fkadj_server *s);
/* Copies the request; returns at once with its id. */
fkadj_status fkadj_server_submit(fkadj_server *s, const fkadj_params *p, double dt, int nt,
                                 const int *active_index, int nrows, int ncols, int n_num,
                                 const double *gh_num, const double *gamma, int64_t S_ncol,
                                 const int64_t *S_colptr, const int64_t *S_rowidx, const double *S_val,
                                 double alpha, const double *Et, const double *y_ini, int want_grad,
                                 int64_t *request_id);
/* 1 done, 0 queued or running, -2 failed, -1 unknown id. */
int fkadj_server_poll(fkadj_server *s, int64_t request_id);
/* Waits at most timeout_s seconds (FKADJ_ERR_TIMEOUT when it expires). */
fkadj_status fkadj_server_wait(fkadj_server *s, int64_t request_id, double timeout_s);
/* Results of a finished request, then forgets it.  latency_s[0] = submit to
 * done, latency_s[1] = submit to admission (may be NULL). */
fkadj_status fkadj_server_result(fkadj_server *s, int64_t request_id, double *L0, double *LE, double *Lcost,
                                 double *gradE, int64_t n_gradE, double latency_s[2]);
/* out: completed, failed, queued, running, peak running, device bytes reserved. */
void fkadj_server_stats(fkadj_server *s, int64_t out[6]);

/* ------------------------------------------------------------------------
 * z.gh without allocating.  No counterpart in the reference: it is the
 * reduction the reference takes once per backward step (sum of z_u * gh over
 * the grid, NaN terms skipped), offered to callers that cannot call
 * cudaMalloc -- their device memory belongs to another allocator or pool, or
 * they must not pay cudaMalloc/cudaFree inside a timed loop.
 *   d_zu, d_gh  device arrays, dense row-major nrows x ncols (NaN at holes)
 *   d_out       device double that receives the sum (written on `stream`)
 * The partial sums use a fixed device array of FKADJ_NOALLOC_MAX_SUBBLOCKS
 * 16x16 sub-blocks (512 KiB, held by every GPU that loads the library until
 * exit); larger grids are rejected with FKADJ_ERR_ARG.  The first call on a
 * device resolves that array's address (make it before any stream capture)
 * and the library keeps it for the life of the process: after cudaDeviceReset,
 * or anything else that re-creates the device's primary context, it is stale
 * and the entry point must not be called again in that process.
 * All calls on a device share the array: calls that overlap on the GPU race,
 * so the caller serialises them.  Nothing is allocated.
 * --------------------------------------------------------------------- */
#define FKADJ_NOALLOC_MAX_SUBBLOCKS 65536
fkadj_status fkadj_zgh_dot_noalloc(const double *d_zu, const double *d_gh, int nrows, int ncols, double *d_out,
                                   void *stream);

#ifdef __cplusplus
}
#endif
#endif /* FKADJ_H */
