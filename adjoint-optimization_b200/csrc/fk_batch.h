// fk_batch.h -- many independent FK problems advanced together.
//
// Each job (one objective or one gradient of one resident Problem) is a fixed
// program of actions: nt forward steps, the objective at T, the backward sweep
// (with sqrt-checkpoint segment recomputes), and a final reduction.  A tick
// takes the next action of every active job and runs them as at most three
// launches -- all forward-type steps, all midpoint steps, all adjoint steps of
// every job -- through the batched persistent kernels (k_batch_*), whose work
// queues reach the device in one small copy per tick.  Jobs of different grid
// sizes and horizons therefore
// share every launch, small grids fill the GPU together, and a job finishing or
// starting changes only the next tick's queue.  The reference has no batching
// (one instance per MATLAB call, simple_grad_desc.m:82).
#pragma once

#include <cstdint>
#include <memory>
#include <array>
#include <vector>

#include <cuda_runtime.h>

#include "fk_engine.h"

namespace fkadj {

struct Action {
    enum Kind : uint8_t { FWD, OBJ, RECOMP, ADJ, EXADJ, FINISH } kind;
    int idx;
};

struct Job {
    int id = -1;
    int prob = -1;
    bool want_grad = true;
    std::vector<Action> plan;
    size_t pc = 0;
    TrajPlan tp{};
    double* cur = nullptr;  // forward sweep: current state
    double* yT = nullptr;
    double *z = nullptr, *z2 = nullptr;
    int cur_c = 0;
    bool have_fcarry = false, have_jcarry = false;  // f(y) / J(y) carried from the previous backward step
    bool finishing = false, done = false;
    fkadj_status status = FKADJ_OK;
    double* h_out = nullptr;  // pinned: [0] sum for L0, [1..rows] reductions
    size_t h_cap = 0;         // doubles in h_out (a buffer of the engine's pool)
    int rows = 0;
    cudaEvent_t ev = nullptr;
    std::vector<double> Et;
    double L0 = 0, LE = 0, Lcost = 0;
    std::vector<double> gradE;
    double t_submit = 0, t_start = 0, t_done = 0;  // host seconds
};

class BatchEngine {
public:
    ~BatchEngine();
    fkadj_status init(const fkadj_options* opt);

    // Resident problems live on the engine's stream; ids are dense from 0.
    fkadj_status add_problem(const fkadj_params& p, double dt, int nt, const int* active_index, int nrows,
                             int ncols, int n_num, const double* gh_num, const double* gamma, int64_t S_ncol,
                             const int64_t* S_colptr, const int64_t* S_rowidx, const double* S_val, double alpha,
                             int grad_mode, int ckpt_policy, int64_t ckpt_budget, int* id);
    fkadj_status remove_problem(int id);

    // Queues a job; the initial state is uploaded now (y_ini may be null to
    // re-use the problem's resident one).  Jobs start at the next tick.
    fkadj_status submit(int prob, const double* Et, const double* y_ini, bool want_grad, int* job_id);

    // One tick; returns the number of jobs still running or queued.
    fkadj_status tick(int* active);
    fkadj_status run_all();

    bool job_done(int job) const;
    fkadj_status job_result(int job, double* L0, double* LE, double* Lcost, double* gradE, int64_t n_gradE);
    fkadj_status release_job(int job);
    const Job* job(int id) const;

    int64_t launches() const { return launches_; }
    int64_t ticks() const { return ticks_; }
    cudaStream_t stream() const { return st_; }
    int tile(int kind) const { return tiles_[kind]; }
    int64_t device_bytes() const;
    Problem* problem(int id) { return (id >= 0 && id < (int)probs_.size()) ? probs_[id].get() : nullptr; }

private:
    fkadj_status fail(cudaError_t e, const char* what);
    fkadj_status build_plan(Job& j);
    fkadj_status host_action(Job& j, const Action& a);
    fkadj_status tick_action(Job& j, const Action& a);
    fkadj_status finish_poll(Job& j);
    fkadj_status sync_instances();

    cudaStream_t st_ = nullptr;
    bool own_stream_ = false;
    cudaMemPool_t pool_ = nullptr;  // device memory of the engine's problems
    int tiles_[4] = {0, 0, 0, 0};  // fwd, mid, adj presets; fused preset (fused_shape)
    int adj_path_ = 0;             // reference-adjoint path (Problem::AdjPath), from the autotuner
    bool tuned_ = false;        // presets fixed (options.tile > 0) or autotuned
    HermiteW hw_{};
    std::vector<std::unique_ptr<Problem>> probs_;
    std::vector<BatchInstance> inst_host_;
    DevBuf inst_dev_;
    bool inst_dirty_ = true;
    std::vector<std::unique_ptr<Job>> jobs_;
    std::vector<int> active_;  // job ids in tick order
    static constexpr int kQueueRing = 64;
    BatchItem* qring_ = nullptr;        // pinned: kQueueRing slots of 4 x kBatchMaxItems items
    cudaEvent_t qev_[kQueueRing] = {};  // a slot's copy has run
    uint64_t qcount_ = 0;
    DevBuf qdev_;                       // the device queue the kernels read
    BatchTick* t_fwd_ = nullptr;  // host staging of the four queues
    BatchTick* t_mid_ = nullptr;
    BatchTick* t_adj_ = nullptr;
    BatchTick* t_fus_ = nullptr;  // fused reference-adjoint steps
    int64_t launches_ = 0, ticks_ = 0;
    fkadj_options opt_{};
    // Blocks of ticks: while no running job needs host work (its objective or
    // its results), up to kBlockMax ticks are planned at once, their queues
    // uploaded in one copy, and their launches replayed from a CUDA graph
    // captured once per (ticks, kinds present) that reads each queue's size
    // and place from a header in device memory.  FKADJ_BATCH_GRAPHS=0 keeps
    // one tick at a time.
    static constexpr int kBlockMax = 32;
    static constexpr int kBlockRing = 4;
    bool block_graphs_ = true;
    char* bring_ = nullptr;             // pinned staging: kBlockRing slots of block_bytes()
    cudaEvent_t bev_[kBlockRing] = {};  // a slot's copy has run
    uint64_t bcount_ = 0;
    DevBuf bdev_;                       // the device block: headers, then items
    // (ticks, kind mask, preset of each kind) -> graph: the presets are part of
    // the key because a graph's launches are fixed at capture, while the
    // engine cuts its queues into tiles of the current presets (the autotuner
    // sets them at the first tick with a gradient job, after blocks of
    // objective-only ticks may have been captured with the default presets)
    std::vector<std::pair<std::array<int, 6>, cudaGraphExec_t>> bgraphs_;
    static size_t block_hdr_bytes() { return (size_t)kBlockMax * 4 * 4 * sizeof(int); }
    static size_t block_bytes() { return block_hdr_bytes() + sizeof(BatchItem) * (size_t)kBlockMax * 4 * kBatchMaxItems; }
    int device_run(const Job& j) const;  // device actions before the job's next host action
    fkadj_status launch_block(int K, const std::vector<int>& ready);
    fkadj_status launch_tick();
    // Pinned result buffers, reused across jobs: cudaFreeHost synchronises the
    // device, which would stall every running job each time one finishes.
    std::vector<std::pair<size_t, double*>> pinned_free_;
    double* take_pinned(size_t n, size_t* cap);
    void give_pinned(double* p, size_t cap);
};

double host_seconds();

}  // namespace fkadj
