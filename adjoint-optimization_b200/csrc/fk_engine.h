// fk_engine.h -- resident FK problem: geometry, objective, work buffers and
// the trajectory store of one instance on one GPU, plus the forward and
// gradient drivers (the roles of fk_forward_Et_comp, cu-F:646-849, and
// fk_grad_Et_comp, cu-G:1569-1938).
#pragma once

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/fkadj.h"
#include "fk_kernels.h"
#include "fk_spline.h"

namespace fkadj {

void set_error(const std::string& msg);

// One device allocation released on destruction.  With a memory pool set
// (problems owned by a batch engine) allocation and release are stream-ordered
// on `st`: releasing needs no device synchronisation, so a finished request can
// free its memory while the others keep running.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaStream_t st = nullptr;
    cudaMemPool_t pool = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) {
            if (pool) cudaFreeAsync(p, st);
            else cudaFree(p);
        }
        p = nullptr;
        bytes = 0;
    }
    cudaError_t alloc(size_t b) {
        release();
        if (b == 0) return cudaSuccess;
        cudaError_t e = pool ? cudaMallocFromPoolAsync(&p, b, pool, st) : cudaMalloc(&p, b);
        if (e == cudaSuccess) bytes = b;
        else p = nullptr;
        return e;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

struct Timing {
    double fwd_ms = 0, bwd_ms = 0, total_ms = 0;
};

// Where the states y(t_i) live during one gradient.
struct TrajPlan {
    int policy = FKADJ_CKPT_FULL;  // resolved policy (FULL / SQRT / BINOMIAL)
    int stride = 1;                // steps between stored states (SQRT)
    int nslots = 0;                // stored state slots
    int seg_slots = 0;             // recompute buffer slots
    bool keep_f = false;           // k1 = f(y_t, Et[t]) kept beside the states the
                                   // backward sweep walks (FULL: all, SQRT: the segment)
    int64_t recompute = 0;         // forward steps the backward sweep recomputes
};

class BatchEngine;

class Problem {
    friend class BatchEngine;

public:
    ~Problem();
    fkadj_status init(const fkadj_params& p, double dt, int nt, const int* active_index, int nrows,
                      int ncols, int n_num, const double* gh_num, const double* gamma, int64_t S_ncol,
                      const int64_t* S_colptr, const int64_t* S_rowidx, const double* S_val, double alpha,
                      const fkadj_options* opt, bool need_objective);

    fkadj_status forward(const double* Et, const double* y_ini, int nstep, int ns, double* ys, double* yf);
    fkadj_status objective(const double* Et, const double* y_ini, double* L0, double* LE, double* Lcost,
                           double* yf);
    fkadj_status grad(const double* Et, const double* y_ini, double* L0, double* LE, double* Lcost,
                      double* gradE, double* yf);

    int64_t device_bytes() const;
    // Device bytes a problem of this size will hold once a job has run
    // (geometry, work states, adjoint work, Jacobian caches, trajectory store
    // under `policy`), for admission control before anything is allocated.
    static int64_t estimate_bytes(int nrows, int ncols, int nt, int n_num, int64_t nnz, int grad_mode,
                                  int policy, bool want_grad);
    Timing last_timing() const { return timing_; }
    // trajectory plan of the last gradient (policy FULL/SQRT/BINOMIAL, 0 = none yet)
    const TrajPlan& last_plan() const { return traj_plan_; }
    bool has_trajectory() const { return traj_.p != nullptr; }
    int64_t last_launches() const { return launches_; }

    // Sampled per-kernel device times (CUDA events around every k-th launch
    // of each kernel kind; off by default).
    enum Kernel { K_FWD = 0, K_MID = 1, K_ADJ = 2, K_COUNT = 3 };
    void set_profiling(bool on) { profiling_ = on; }
    void kernel_time(int k, double* avg_ms, int64_t* samples) const;
    const DevGrid& grid() const { return g_; }
    int nt() const { return nt_; }
    int n_num() const { return n_num_; }
    cudaStream_t stream() const { return st_; }
    // tile preset per kernel kind; chosen by autotune() unless fixed by options
    enum TileKind { T_FWD = 0, T_MID = 1, T_ADJ = 2, T_EXACT = 3 };
    // reference-mode backward step: k_adj_mid + k_adj_step, or k_adj_fused
    // reading the cached J_F(y_i)^T, or k_adj_fused evaluating it
    enum AdjPath { ADJ_SPLIT = 0, ADJ_FUSED = 1, ADJ_FUSED_RECOMPUTE = 2 };
    int adjoint_path() const { return adj_path_; }
    int fused_tile() const { return tkf_; }
    // Stream-ordered device memory from `pool` (call before init).
    void use_pool(cudaMemPool_t pool) { pool_ = pool; }
    // A problem of a one-shot entry point (call before init): device memory
    // from `pool` (null: cudaMalloc), pinned staging from the process's cache.
    void set_oneshot(cudaMemPool_t pool) {
        pool_ = pool;
        oneshot_ = true;
    }
    int tile(int kind) const { return tk_[kind]; }
    void set_tile(int kind, int t) { tk_[kind] = t; }
    // rows per tile in use for a kernel kind (the preset's height, or fewer
    // when the autotuner found a one-wave split faster)
    // rows per tile of a kernel kind as launched (the adjoint step takes its
    // rows on the row-segment lattice only)
    int tile_rows(int kind) const {
        return ty_[kind] > 0 && (kind != T_ADJ || segs_) ? ty_[kind] : tile_shape(tk_[kind]).ty;
    }
    // Times every tile preset of every kernel kind on the current initial
    // state (a few launches each) and keeps the fastest per kind.  Results do
    // not depend on the choice (fixed-order reductions).
    fkadj_status autotune();
    fkadj_status autotune_trials();

    // Lower-level pieces (used by the batch / serving layers and the tests).
    // upload_state with y_ini == nullptr re-uses the initial state of the
    // previous call (kept resident on the device).
    fkadj_status upload_state(const double* y_ini, double* d_state);
    // Spline samples of Et on the host; with upload, also the device tables the
    // standalone kernels read (the batched kernels take E by value).
    fkadj_status prepare_E(const double* Et, bool upload = true);
    fkadj_status step_forward(int i, const double* yin, double* yout, double* k1 = nullptr);
    double* state_buf(int k) const { return work_.as<double>() + (size_t)k * state_elems(); }
    size_t state_elems() const { return (size_t)3 * g_.plane; }
    size_t state_bytes() const { return state_elems() * sizeof(double); }

private:
    fkadj_status fail_cuda(cudaError_t e, const char* what);
    // brackets a launch of kernel kind k with sampled events when profiling
    cudaError_t prof_begin(int k);
    cudaError_t prof_end(int k);
    fkadj_status prof_collect();
    // FKADJ_ERR_TIMEOUT when a kernel's bounded wait expired since the last check
    fkadj_status check_fault();
    // Resolves the checkpoint policy.  AUTO takes FULL when the budget holds
    // every state, else whichever of SQRT and BINOMIAL fits and recomputes
    // fewer forward steps (costed in forward-step equivalents, the binomial
    // reference-mode reversal's extra per-step work, measured at 0.9 of a
    // forward step, included); with
    // sqrt_or_full_only (the batch engine, which runs no binomial schedule)
    // BINOMIAL only when SQRT does not fit.
    fkadj_status plan_trajectory(TrajPlan& tp, bool sqrt_or_full_only = false);
    fkadj_status ensure_traj(const TrajPlan& tp);
    fkadj_status run_objective(const double* yT, double* L0);
    fkadj_status objective_async(const double* yT);
    fkadj_status grad_exact_backward(const TrajPlan& tp, double* lam, double* lam2);
    fkadj_status advance(int a, int m, const double* src, double* dst);
    fkadj_status reverse_binomial(int nt, double* y0, std::vector<double*>& free,
                                  const std::function<fkadj_status(int, const double*)>& visit);
    // all_rows: keep the z.gh partials of every step (the batch engine);
    // otherwise a window of kPartialWindow rows reduced as the sweep goes.
    fkadj_status ensure_adjoint_work(bool all_rows = false);
    // z.gh partial row `row` of group g (exact mode: 3 groups of nt rows;
    // reference mode: one group of nt+1 rows) in the window
    double* prow(int g, int row) const {
        return partial_.as<double>() + ((size_t)g * pwin_ + (size_t)(row % pwin_)) * nsb_;
    }
    // reduces the rows row .. row+pwin-1 (clipped to rows_g) of group g into zgh
    cudaError_t flush_rows(int g, int row, int rows_g);
    cudaError_t flush_range(int g, int row0, int n);
    static constexpr int kPartialWindow = 512;
    fkadj_status download_grid(const double* d_state, double* host_dense);
    double* slot(int k) const { return traj_.as<double>() + (size_t)k * state_elems(); }
    double* segslot(int k) const { return seg_.as<double>() + (size_t)k * state_elems(); }
    double* fslot(int k) const { return kf_.as<double>() + (size_t)k * state_elems(); }
    // E samples of step i read from the device tables (uploaded by prepare_E)
    const double* etab() const { return Ed_.as<double>(); }
    EStep efwd(int i) const {
        const double* t = etab();
        return EStep::table(t + i, t + (nt_ + 1) + i, t + i + 1);  // Et[i], E(t_i + dt/2), Et[i+1]
    }
    EStep emid(int i) const {
        const double* t = etab();
        return EStep::table(t + i - 1, t + i, t + (2 * nt_ + 1) + i - 1);  // Et[i-1], Et[i], E(t_{i-1} + dt/3)
    }
    // The gradient's device work after the initial state is in place: forward
    // sweep, objective, backward sweep, reductions, and the copies of L0 and the
    // z.gh rows into pinned host memory.  Issued directly or captured once into a
    // CUDA graph and replayed (use_graph).
    fkadj_status grad_sequence(const TrajPlan& tp, bool exact, double** yT);
    fkadj_status grad_replay(const TrajPlan& tp, bool exact, double** yT);
    // segment graphs of a gradient run as plain launches (fk_engine.cu)
    bool segment_graphs_wanted() const;
    fkadj_status segment_begin();
    fkadj_status segment_launch();
    void segment_abort();
    void drop_segment_graphs();
    cudaGraphExec_t seg_exec_[2] = {nullptr, nullptr};
    cudaEvent_t seg_done_[2] = {nullptr, nullptr};
    int seg_next_ = 0;
    bool seg_on_ = false;
    void drop_graph();

    fkadj_params p_{};
    DevModel P_{};
    DevGrid g_{};
    HermiteW hw_{};
    double dt_ = 0, alpha_ = 0, gamma_[3] = {0, 0, 0};
    int nt_ = 0, n_num_ = 0, device_ = 0, nsbx_ = 0, nsby_ = 0, nsb_ = 0;
    // z.gh partials on the row-segment lattice (nsb_ = nsbx_ x nrows; the
    // adjoint step's tiles then take balanced rows) instead of the 16x16 one
    // (nsb_ = nsbx_ x nsby_); chosen by ensure_adjoint_work
    bool segs_ = false;
    int tk_[4] = {0, 0, 0, 0};  // tile preset per kernel kind (TileKind)
    int tkf_ = 0;               // fused reference-adjoint preset (fused_shape)
    int adj_path_ = 0;          // AdjPath of the reference-mode backward step
    int forced_path_ = -1;      // AdjPath fixed by FKADJ_ADJ_PATH (-1: autotuned)
    // Jacobian caches of the split backward step (FKADJ_JCACHE): 2 = J(yh)
    // from the midpoint kernel and J(y_{i-1}) carried to the next step; 1 =
    // the carry only, the step evaluates J(yh); 0 = the step evaluates both
    int jcache_mode_ = 2;
    int ty_[4] = {0, 0, 0, 0};  // rows per tile per kind (0 = the preset's height)
    bool autotune_ = true, tuned_ = false, tuned_fwd_ = false;
    bool tiles_fixed_ = false;  // FKADJ_TILES fixed every kind's preset: autotune() keeps them
    bool own_stream_ = false, have_obj_ = false;
    cudaMemPool_t pool_ = nullptr;
    int verbose_ = 0;
    int grad_mode_ = FKADJ_GRAD_REF, ckpt_policy_ = FKADJ_CKPT_AUTO;
    int64_t ckpt_budget_ = 0;
    cudaStream_t st_ = nullptr;
    cudaEvent_t ev_[3] = {nullptr, nullptr, nullptr};

    // device buffers
    DevBuf gh_, wc_, pos_, Srow_, Scol_, Sval_, yc_, zc_, opart_, osum_;
    DevBuf fcode_;     // forward stencil codes (uint8 per padded cell; unset when the NaN tests decide)
    DevBuf fault_;     // this problem's fault word: set by a step kernel whose bounded wait expired
    unsigned* fault() const { return fault_.as<unsigned>(); }
    DevBuf work_;      // 4 states: two ping-pong, z pair is separate
    DevBuf zbuf_;      // 2 adjoint states
    DevBuf yh_;        // midpoint state
    DevBuf partial_;   // (nt+1) x ntiles zgh partials
    DevBuf zgh_;       // nt+1
    DevBuf traj_, seg_;
    DevBuf kf_;        // kept k1 = f(y_t) per stored / recomputed state (TrajPlan::keep_f)
    DevBuf y0res_;     // resident initial state
    DevBuf stg_;       // stage states Y2, Y3, Y4 of one step (exact mode)
    DevBuf jcache_;    // cached Jacobians (reference mode): J(y) ping-pong + J(yh)
    DevBuf fcache_;    // f(y) carried between backward steps (reference mode)
    DevBuf Ed_;        // E tables: Et (nt+1), E at half steps (nt), E at third steps (nt)
    double* Ehost_ = nullptr;  // pinned staging of the E tables
    double* hres_ = nullptr;   // pinned results: L0 partial sum, then the z.gh rows
    size_t hres_n_ = 0;
    size_t Ehost_n_ = 0;       // capacity of Ehost_ (doubles)
    bool oneshot_ = false;
    bool have_y0_ = false;

    // captured gradient sequence
    struct GraphKey {
        int policy = -1, nslots = 0, seg_slots = 0, keep_f = 0, exact = 0, gen = 0, path = 0, tkf = 0;
        int tk[4] = {0, 0, 0, 0}, ty[4] = {0, 0, 0, 0};
        bool operator==(const GraphKey& o) const;
    };
    bool graphs_ = true;         // FKADJ_NO_GRAPHS=1 in the environment turns replay off
    cudaGraphExec_t gexec_ = nullptr;
    GraphKey gkey_{};
    GraphKey seen_key_{};        // configuration of the previous gradient
    GraphKey graph_key(const TrajPlan& tp, bool exact) const;
    int64_t glaunches_ = 0;
    double* gyT_ = nullptr;
    int buf_gen_ = 0;            // bumped whenever a buffer the sequence uses is reallocated
    int pwin_ = 1;               // rows per group in the z.gh partial window
    bool capturing_ = false;
    TrajPlan traj_plan_{};

    // sampled kernel timing
    bool profiling_ = false;
    int prof_every_ = 1;
    int64_t kcount_[K_COUNT] = {0, 0, 0};
    int64_t ksamples_[K_COUNT] = {0, 0, 0};
    double kms_[K_COUNT] = {0, 0, 0};
    struct ProfRec {
        int k;
        cudaEvent_t a, b;
    };
    std::vector<ProfRec> prof_pool_;
    size_t prof_used_ = 0;
    bool prof_open_ = false;

    // host
    std::vector<double> Et_, ypp_, Eh_, E3_;
    NakSpline* spline_ = nullptr;
    Timing timing_{};
    int64_t launches_ = 0;
};

// The binomial schedule's first chain of checkpoints (the states the forward
// sweep stores), and the forward steps its reversal then recomputes.
std::vector<int> binomial_spine(int nt, int free_slots);
int64_t binomial_recompute_steps(int nt, int free_slots);

// Memory the one-shot entry points keep between calls: the per-device pool
// (null when FKADJ_ONESHOT_POOL=0) and its release (fkadj_release_cached_memory).
cudaMemPool_t oneshot_pool(const fkadj_options* opt);
fkadj_status release_oneshot_memory();

}  // namespace fkadj
