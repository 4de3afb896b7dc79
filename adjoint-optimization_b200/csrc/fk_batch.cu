// fk_batch.cu -- see fk_batch.h.
#include "fk_batch.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace fkadj {

HermiteW hermite_weights();

double host_seconds() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

#define BCK(call, what)                                 \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return fail(e_, what);   \
    } while (0)

fkadj_status BatchEngine::fail(cudaError_t e, const char* what) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? FKADJ_ERR_NOMEM : FKADJ_ERR_CUDA;
}

BatchEngine::~BatchEngine() {
    if (st_) cudaStreamSynchronize(st_);
    for (auto& j : jobs_) {
        if (!j) continue;
        if (j->ev) cudaEventDestroy(j->ev);
        if (j->h_out) cudaFreeHost(j->h_out);
    }
    for (auto& f : pinned_free_) cudaFreeHost(f.second);
    pinned_free_.clear();
    jobs_.clear();
    probs_.clear();  // their buffers go back to the pool in stream order
    if (pool_) {
        if (st_) cudaStreamSynchronize(st_);
        cudaMemPoolDestroy(pool_);
    }
    cudaFreeHost(t_fwd_);
    cudaFreeHost(t_mid_);
    cudaFreeHost(t_adj_);
    cudaFreeHost(t_fus_);
    for (auto& e : qev_)
        if (e) cudaEventDestroy(e);
    for (auto& e : bev_)
        if (e) cudaEventDestroy(e);
    for (auto& g : bgraphs_) cudaGraphExecDestroy(g.second);
    if (bring_) cudaFreeHost(bring_);
    if (qring_) cudaFreeHost(qring_);
    if (own_stream_ && st_) cudaStreamDestroy(st_);
}

fkadj_status BatchEngine::init(const fkadj_options* opt) {
    fkadj_default_options(&opt_);
    if (opt) opt_ = *opt;
    if (opt_.device >= 0) BCK(cudaSetDevice(opt_.device), "cudaSetDevice");
    if (opt_.stream) {
        st_ = static_cast<cudaStream_t>(opt_.stream);
    } else {
        BCK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking), "cudaStreamCreate");
        own_stream_ = true;
    }
    const int t = batch_preset((opt_.tile > 0 && opt_.tile <= tile_count()) ? opt_.tile - 1 : 0);
    tiles_[0] = tiles_[1] = tiles_[2] = t;
    tiles_[3] = 0;
    // the split midpoint + step kernels unless the autotuner (or FKADJ_ADJ_PATH) picks the fused step
    adj_path_ = Problem::ADJ_SPLIT;
    if (const char* ap = getenv("FKADJ_ADJ_PATH")) {
        if (!std::strcmp(ap, "fused")) adj_path_ = Problem::ADJ_FUSED;
        else if (!std::strcmp(ap, "fused-recompute")) adj_path_ = Problem::ADJ_FUSED_RECOMPUTE;
    }
    if (const char* ft = getenv("FKADJ_FUSED_TILE")) {
        const int f = std::atoi(ft);
        if (f >= 0 && f < fused_count()) tiles_[3] = f;
    }
    tuned_ = opt_.tile > 0 && opt_.tile <= tile_count();
    hw_ = hermite_weights();
    {
        // the problems' device memory: a pool of this engine, allocated and
        // freed in stream order, kept reserved between requests
        int dev = 0;
        BCK(cudaGetDevice(&dev), "cudaGetDevice");
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        BCK(cudaMemPoolCreate(&pool_, &props), "memory pool");
        uint64_t keep = UINT64_MAX;
        BCK(cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep), "memory pool");
    }
    BCK(cudaMallocHost(&qring_, sizeof(BatchItem) * (size_t)kQueueRing * 4 * kBatchMaxItems), "queue ring");
    BCK(qdev_.alloc(sizeof(BatchItem) * 4 * kBatchMaxItems), "device queue");
    BCK(cudaMallocHost(&t_fwd_, sizeof(BatchTick)), "pinned tick");
    BCK(cudaMallocHost(&t_mid_, sizeof(BatchTick)), "pinned tick");
    BCK(cudaMallocHost(&t_adj_, sizeof(BatchTick)), "pinned tick");
    BCK(cudaMallocHost(&t_fus_, sizeof(BatchTick)), "pinned tick");
    {
        const char* bg = getenv("FKADJ_BATCH_GRAPHS");
        block_graphs_ = !(bg && bg[0] == '0') && st_ != nullptr && st_ != cudaStreamLegacy &&
                        st_ != cudaStreamPerThread;
    }
    if (block_graphs_) {
        BCK(cudaMallocHost(&bring_, block_bytes() * kBlockRing), "pinned block staging");
        BCK(bdev_.alloc(block_bytes()), "device block");
    }
    return FKADJ_OK;
}

fkadj_status BatchEngine::add_problem(const fkadj_params& p, double dt, int nt, const int* ai, int nrows, int ncols,
                                      int n_num, const double* gh_num, const double* gamma, int64_t S_ncol,
                                      const int64_t* S_colptr, const int64_t* S_rowidx, const double* S_val,
                                      double alpha, int grad_mode, int ckpt_policy, int64_t ckpt_budget, int* id) {
    fkadj_options o = opt_;
    o.stream = st_;
    o.grad_mode = grad_mode;
    o.ckpt_policy = ckpt_policy;
    o.ckpt_budget_bytes = ckpt_budget;
    o.tile = tiles_[0] + 1;  // fixed preset: no per-problem autotune inside a batch
    auto pb = std::make_unique<Problem>();
    pb->use_pool(pool_);
    const bool need_obj = gamma && S_colptr;
    fkadj_status s = pb->init(p, dt, nt, ai, nrows, ncols, n_num, gh_num, gamma, S_ncol, S_colptr, S_rowidx,
                              S_val, alpha, &o, need_obj);
    if (s) return s;
    BatchInstance bi;
    bi.P = pb->P_;
    bi.g = pb->g_;
    bi.gh = pb->gh_.as<double>();
    bi.wc = pb->wc_.as<uint8_t>();
    bi.fault = pb->fault();
    bi.nsbx = pb->nsbx_;
    int slot = -1;
    for (size_t k = 0; k < probs_.size(); ++k)
        if (!probs_[k]) {
            slot = (int)k;
            break;
        }
    if (slot < 0) {
        slot = (int)probs_.size();
        probs_.emplace_back();
        inst_host_.emplace_back();
    }
    probs_[slot] = std::move(pb);
    inst_host_[slot] = bi;
    inst_dirty_ = true;
    *id = slot;
    return FKADJ_OK;
}

fkadj_status BatchEngine::remove_problem(int id) {
    if (id < 0 || id >= (int)probs_.size() || !probs_[id]) {
        set_error("unknown problem id");
        return FKADJ_ERR_ARG;
    }
    for (int a : active_)
        if (jobs_[a]->prob == id) {
            set_error("problem has a running job");
            return FKADJ_ERR_BUSY;
        }
    probs_[id].reset();  // stream-ordered release: no synchronisation
    return FKADJ_OK;
}

fkadj_status BatchEngine::sync_instances() {
    const size_t b = inst_host_.size() * sizeof(BatchInstance);
    if (inst_dev_.bytes < b) {
        BCK(cudaStreamSynchronize(st_), "synchronize");
        BCK(inst_dev_.alloc(std::max(b, (size_t)64 * sizeof(BatchInstance))), "alloc instance table");
    }
    BCK(cudaMemcpyAsync(inst_dev_.p, inst_host_.data(), b, cudaMemcpyHostToDevice, st_), "upload instance table");
    inst_dirty_ = false;
    return FKADJ_OK;
}

int64_t BatchEngine::device_bytes() const {
    int64_t s = (int64_t)inst_dev_.bytes;
    for (auto& p : probs_)
        if (p) s += p->device_bytes();
    return s;
}

fkadj_status BatchEngine::build_plan(Job& j) {
    Problem& P = *probs_[j.prob];
    const int nt = P.nt_;
    j.plan.clear();
    j.plan.reserve((size_t)3 * nt + 4);
    for (int k = 0; k < nt; ++k) j.plan.push_back({Action::FWD, k});
    j.plan.push_back({Action::OBJ, 0});
    if (j.want_grad) {
        const bool exact = P.grad_mode_ == FKADJ_GRAD_EXACT;
        const int c = j.tp.stride, K = j.tp.nslots - 1;
        if (j.tp.policy == FKADJ_CKPT_FULL) {
            if (exact)
                for (int t = nt - 1; t >= 0; --t) j.plan.push_back({Action::EXADJ, t});
            else
                for (int i = nt; i > 0; --i) j.plan.push_back({Action::ADJ, i});
        } else {
            for (int k = K - 1; k >= 0; --k) {
                const int s0 = k * c, s1 = std::min(s0 + c, nt);
                for (int t = s0; t < s1 - 1; ++t) j.plan.push_back({Action::RECOMP, t});
                if (exact)
                    for (int t = s1 - 1; t >= s0; --t) j.plan.push_back({Action::EXADJ, t});
                else
                    for (int i = s1; i > s0; --i) j.plan.push_back({Action::ADJ, i});
            }
        }
        j.rows = exact ? 3 * nt : nt + 1;
    } else {
        j.rows = 0;
    }
    j.plan.push_back({Action::FINISH, 0});
    j.pc = 0;
    return FKADJ_OK;
}

fkadj_status BatchEngine::submit(int prob, const double* Et, const double* y_ini, bool want_grad, int* job_id) {
    if (prob < 0 || prob >= (int)probs_.size() || !probs_[prob]) {
        set_error("unknown problem id");
        return FKADJ_ERR_ARG;
    }
    for (int a : active_)
        if (jobs_[a]->prob == prob) {
            set_error("problem already has a running job");
            return FKADJ_ERR_BUSY;
        }
    if ((int)active_.size() >= kBatchMaxItems) {
        set_error("batch is full");
        return FKADJ_ERR_BUSY;
    }
    Problem& P = *probs_[prob];
    if (want_grad && !P.have_obj_) {
        set_error("problem has no objective");
        return FKADJ_ERR_ARG;
    }
    auto j = std::make_unique<Job>();
    j->id = (int)jobs_.size();
    j->prob = prob;
    j->want_grad = want_grad;
    j->t_submit = host_seconds();
    fkadj_status s;
    if ((s = P.prepare_E(Et, false))) return s;  // batched kernels take E by value
    j->Et.assign(Et, Et + P.nt_ + 1);
    if (want_grad) {
        if ((s = P.plan_trajectory(j->tp, true))) return s;
        if (j->tp.policy == FKADJ_CKPT_BINOMIAL) {
            set_error("batched jobs store full or sqrt trajectories; the binomial schedule runs in the "
                      "standalone engine (raise ckpt_budget_bytes or use fkadj_problem_grad)");
            return FKADJ_ERR_NOMEM;
        }
        // k1 = f(y) kept by the segment recompute (sqrt store, reference mode);
        // the full store evaluates it (keeping it there doubles the store)
        if (j->tp.policy != FKADJ_CKPT_SQRT) j->tp.keep_f = false;
        if ((s = P.ensure_traj(j->tp))) return s;
        if ((s = P.ensure_adjoint_work(true))) return s;  // the batch reduces all rows at the end
        if ((s = P.upload_state(y_ini, P.slot(0)))) return s;
        j->cur = P.slot(0);
        j->z = P.zbuf_.as<double>();
        j->z2 = j->z + P.state_elems();
    } else {
        j->tp.policy = 0;
        if ((s = P.upload_state(y_ini, P.state_buf(0)))) return s;
        j->cur = P.state_buf(0);
    }
    if ((s = build_plan(*j))) return s;
    j->h_out = take_pinned((size_t)j->rows + 2, &j->h_cap);  // [0] L0 sum, [1..rows], fault word
    if (!j->h_out) {
        set_error("pinned results: out of host memory");
        return FKADJ_ERR_NOMEM;
    }
    BCK(cudaEventCreateWithFlags(&j->ev, cudaEventDisableTiming), "event");
    j->t_start = host_seconds();
    *job_id = j->id;
    active_.push_back(j->id);
    jobs_.push_back(std::move(j));
    return FKADJ_OK;
}

fkadj_status BatchEngine::host_action(Job& j, const Action& a) {
    Problem& P = *probs_[j.prob];
    const size_t nsb = (size_t)P.nsb_;
    if (a.kind == Action::OBJ) {
        fkadj_status s = P.objective_async(j.yT);
        if (s) return s;
        launches_ += 3;
        if (j.want_grad) {
            const bool exact = P.grad_mode_ == FKADJ_GRAD_EXACT;
            BCK(launch_scatter(P.g_, P.zc_.as<double>(), P.n_num_, P.pos_.as<long long>(), exact ? -1.0 : 1.0,
                               j.z, st_),
                "scatter z");
            ++launches_;
            if (!exact) {
                BCK(launch_dot_gh(P.g_, j.z, P.gh_.as<double>(), P.partial_.as<double>() + (size_t)P.nt_ * nsb,
                                  P.nsbx_, P.nsby_, st_),
                    "z.gh");
                ++launches_;
            }
        }
        return FKADJ_OK;
    }
    // FINISH: reductions and results to pinned memory
    if (j.want_grad) {
        BCK(launch_sum_rows(P.partial_.as<double>(), j.rows, P.nsb_, P.zgh_.as<double>(), st_), "reduce");
        ++launches_;
        BCK(cudaMemcpyAsync(j.h_out + 1, P.zgh_.p, sizeof(double) * j.rows, cudaMemcpyDeviceToHost, st_),
            "download");
    }
    BCK(cudaMemcpyAsync(j.h_out, P.osum_.p, sizeof(double), cudaMemcpyDeviceToHost, st_), "download");
    // the problem's fault word after the job's launches (a tile copy whose
    // bounded wait expired), then cleared for the problem's next job
    unsigned* hf = reinterpret_cast<unsigned*>(j.h_out + j.rows + 1);
    *hf = 0;
    BCK(cudaMemcpyAsync(hf, P.fault(), sizeof(unsigned), cudaMemcpyDeviceToHost, st_), "download fault word");
    BCK(cudaMemsetAsync(P.fault(), 0, sizeof(unsigned), st_), "clear fault word");
    BCK(cudaEventRecord(j.ev, st_), "event");
    j.finishing = true;
    return FKADJ_OK;
}

fkadj_status BatchEngine::tick_action(Job& j, const Action& a) {
    Problem& P = *probs_[j.prob];
    const int nt = P.nt_;
    const size_t nsb = (size_t)P.nsb_;
    const int c = j.tp.stride, K = j.tp.nslots - 1;
    const bool full = j.tp.policy == FKADJ_CKPT_FULL;
    // each kernel kind runs its own tile preset: the queue of kind k is cut
    // into tiles of that preset
    auto ntiles = [&](const BatchTick* T, int& ntx) {
        const int k = T == t_fwd_ ? 0 : (T == t_mid_ ? 1 : (T == t_adj_ ? 2 : 3));
        const TileShape ts = k == 3 ? fused_shape(tiles_[3]) : tile_shape(tiles_[k]);
        ntx = (P.g_.ncols + ts.tx - 1) / ts.tx;
        return ntx * ((P.g_.nrows + ts.ty - 1) / ts.ty);
    };
    auto seg = [&](int t, int k) -> double* {  // backward-sweep state store
        if (full) return P.slot(t);
        const int s0 = k * c, s1 = std::min(s0 + c, nt);
        if (t == s0) return P.slot(k);
        if (t == s1) return P.slot(k + 1);
        return P.segslot(t - s0 - 1);
    };
    // k1 = f(y_t) kept by segment k's recompute, for t = s0 .. s1-2
    auto kept = [&](int t, int k) -> double* {
        if (full || !j.tp.keep_f) return nullptr;
        const int s0 = k * c, s1 = std::min(s0 + c, nt);
        return (t >= s0 && t <= s1 - 2) ? P.fslot(t - s0) : nullptr;
    };
    auto push = [&](BatchTick* T, BatchItem it) {
        int ntx = 1;
        const int n = ntiles(T, ntx);
        it.inst = j.prob;
        it.tile0 = T->tiles;
        it.ntx = ntx;
        T->item[T->n++] = it;
        T->tiles += n;
    };
    BatchItem it{};
    switch (a.kind) {
        case Action::FWD: {
            const int k = a.idx;
            double* out;
            if (!j.want_grad) out = (j.cur == P.state_buf(1)) ? P.state_buf(2) : P.state_buf(1);
            else if (full) out = P.slot(k + 1);
            else if ((k + 1) % c == 0) out = P.slot((k + 1) / c);
            else if (k + 1 == nt) out = P.slot(K);
            else out = (j.cur == P.state_buf(1)) ? P.state_buf(2) : P.state_buf(1);
            it.kind = BATCH_FWD;
            it.a = j.cur;
            it.out = out;
            it.E0 = P.Et_[k];
            it.E1 = P.Eh_[k];
            it.E2 = P.Et_[k + 1];
            push(t_fwd_, it);
            j.cur = out;
            if (k + 1 == nt) j.yT = out;
            break;
        }
        case Action::RECOMP: {
            const int t = a.idx, k = t / c;
            it.kind = BATCH_FWD;
            it.a = seg(t, k);
            it.out = seg(t + 1, k);
            it.k1 = kept(t, k);
            it.E0 = P.Et_[t];
            it.E1 = P.Eh_[t];
            it.E2 = P.Et_[t + 1];
            push(t_fwd_, it);
            break;
        }
        case Action::ADJ: {
            const int i = a.idx, k = full ? 0 : (i - 1) / c;
            const size_t pl = (size_t)P.g_.plane;
            double* jy[2] = {P.jcache_.as<double>(), P.jcache_.as<double>() + 7 * pl};
            double* jh = P.jcache_.as<double>() + 14 * pl;
            double* fc[2] = {P.fcache_.as<double>(), P.fcache_.as<double>() + 3 * pl};
            const int nxt = 1 - j.cur_c;
            const double* ya = seg(i - 1, k);
            const double* yb = seg(i, k);
            const double* fa = kept(i - 1, k);
            const double* fb = kept(i, k);
            if (adj_path_ != Problem::ADJ_SPLIT) {  // one fused step
                const bool cache = adj_path_ == Problem::ADJ_FUSED;
                it.kind = BATCH_ADJ_FUSED;
                it.a = j.z;
                it.out = j.z2;
                it.b = yb;
                it.d = ya;
                it.fa = fa;
                it.fin = fb ? fb : (j.have_fcarry ? fc[j.cur_c] : nullptr);
                it.fout = fa ? nullptr : fc[nxt];
                it.E0 = P.Et_[i - 1];
                it.E1 = P.Et_[i];
                it.E2 = P.E3_[i - 1];
                it.row = P.partial_.as<double>() + (size_t)(i - 1) * nsb;
                it.jb = (cache && j.have_jcarry) ? jy[j.cur_c] : nullptr;
                it.ja = cache ? jy[nxt] : nullptr;
                push(t_fus_, it);
                std::swap(j.z, j.z2);
                j.cur_c = nxt;
                j.have_fcarry = fa == nullptr;
                j.have_jcarry = cache;
                break;
            }
            BatchItem m{};
            m.kind = BATCH_MID;
            m.a = ya;
            m.b = yb;
            m.out = P.yh_.as<double>();
            m.E0 = P.Et_[i - 1];
            m.E1 = P.Et_[i];
            m.E2 = P.E3_[i - 1];
            m.fa = fa;
            m.fin = fb ? fb : (j.have_fcarry ? fc[j.cur_c] : nullptr);
            m.fout = fa ? nullptr : fc[nxt];
            m.jh = jh;
            push(t_mid_, m);
            it.kind = BATCH_ADJ_REF;
            it.a = j.z;
            it.out = j.z2;
            it.b = yb;
            it.c = P.yh_.as<double>();
            it.d = ya;
            it.row = P.partial_.as<double>() + (size_t)(i - 1) * nsb;
            it.jb = j.have_jcarry ? jy[j.cur_c] : nullptr;
            it.jh = jh;
            it.ja = jy[nxt];
            push(t_adj_, it);
            std::swap(j.z, j.z2);
            j.cur_c = nxt;
            j.have_fcarry = fa == nullptr;
            j.have_jcarry = true;
            break;
        }
        case Action::EXADJ: {
            const int t = a.idx, k = full ? 0 : t / c;
            double* y = seg(t, k);
            double* stg = P.stg_.as<double>();
            BatchItem f{};
            f.kind = BATCH_FWD;
            f.a = y;
            f.out = P.state_buf(1);
            f.stages = stg;
            f.E0 = P.Et_[t];
            f.E1 = P.Eh_[t];
            f.E2 = P.Et_[t + 1];
            push(t_fwd_, f);
            double* part = P.partial_.as<double>();
            it.kind = BATCH_ADJ_EXACT;
            it.a = j.z;
            it.out = j.z2;
            it.b = y;
            it.stages = stg;
            it.row = part + (size_t)t * nsb;
            it.row2 = part + (size_t)(nt + t) * nsb;
            it.row3 = part + (size_t)(2 * nt + t) * nsb;
            push(t_adj_, it);
            std::swap(j.z, j.z2);
            break;
        }
        default:
            break;
    }
    return FKADJ_OK;
}

fkadj_status BatchEngine::finish_poll(Job& j) {
    const cudaError_t q = cudaEventQuery(j.ev);
    if (q == cudaErrorNotReady) return FKADJ_OK;
    if (q != cudaSuccess) return fail(q, "job completion");
    Problem& P = *probs_[j.prob];
    const int nt = P.nt_;
    const double l0 = -j.h_out[0];
    double le = 0;
    for (int i = 0; i <= nt; ++i) le += j.Et[i] * j.Et[i];
    le *= P.dt_;
    j.L0 = l0;
    j.LE = le;
    j.Lcost = 0.5 * l0 + 0.5 * P.alpha_ * le;
    if (j.want_grad) {
        j.gradE.assign(nt + 1, 0.0);
        const double* r = j.h_out + 1;
        if (P.grad_mode_ == FKADJ_GRAD_EXACT) {
            std::vector<double> gE(nt + 1, 0.0);
            for (int t = 0; t < nt; ++t) {
                gE[t] += r[t];
                gE[t + 1] += r[2 * nt + t];
            }
            NakSpline sp(nt + 1, P.dt_);
            sp.transpose_add(0.5, r + nt, gE.data());
            for (int i = 0; i <= nt; ++i) j.gradE[i] = (gE[i] + P.alpha_ * P.dt_ * j.Et[i]) / P.dt_;
        } else {
            for (int i = 0; i <= nt; ++i) j.gradE[i] = P.alpha_ * j.Et[i] - r[i];
        }
    }
    // the watchdog of the standalone gradient: objective and every gradient entry finite
    bool finite = std::isfinite(l0);
    for (size_t i = 0; finite && i < j.gradE.size(); ++i) finite = std::isfinite(j.gradE[i]);
    j.status = finite ? FKADJ_OK : FKADJ_ERR_NUMERIC;
    if (*reinterpret_cast<const unsigned*>(j.h_out + j.rows + 1)) {
        set_error("a bounded wait in a batched kernel expired (tile copy into shared memory); the job's results "
                  "are invalid");
        j.status = FKADJ_ERR_TIMEOUT;
    }
    j.done = true;
    j.t_done = host_seconds();
    return FKADJ_OK;
}

fkadj_status BatchEngine::tick(int* active) {
    fkadj_status s;
    if (inst_dirty_ && (s = sync_instances())) return s;
    if (!tuned_ && !active_.empty()) {
        // tile presets: the standalone autotuner's choice on the largest job
        int best = -1;
        int64_t cells = -1;
        for (int id : active_) {
            Problem& P = *probs_[jobs_[id]->prob];
            const int64_t c = (int64_t)P.g_.nrows * P.g_.ncols;
            if (jobs_[id]->want_grad && c > cells) cells = c, best = jobs_[id]->prob;
        }
        if (best >= 0) {
            Problem& P = *probs_[best];
            const bool keep = P.autotune_;
            P.autotune_ = true;
            if ((s = P.autotune())) return s;
            P.autotune_ = keep;
            tiles_[0] = batch_preset(P.tk_[Problem::T_FWD]);
            tiles_[1] = batch_preset(P.tk_[Problem::T_MID]);
            tiles_[2] = batch_preset(P.grad_mode_ == FKADJ_GRAD_EXACT ? P.tk_[Problem::T_EXACT]
                                                                       : P.tk_[Problem::T_ADJ]);
            if (P.grad_mode_ == FKADJ_GRAD_REF && P.forced_path_ < 0) {
                adj_path_ = P.adj_path_;
                tiles_[3] = P.tkf_;
            }
            tuned_ = true;
        }
    }
    // finished jobs and host actions first; `ready` jobs have a device action next
    std::vector<int> still, ready;
    still.reserve(active_.size());
    for (int id : active_) {
        Job& j = *jobs_[id];
        if (j.finishing) {
            if ((s = finish_poll(j))) return s;
            if (!j.done) still.push_back(id);
            continue;
        }
        while (j.pc < j.plan.size()) {
            const Action a = j.plan[j.pc];
            if (a.kind != Action::OBJ && a.kind != Action::FINISH) break;
            ++j.pc;
            if ((s = host_action(j, a))) return s;
            if (a.kind == Action::FINISH) break;
        }
        still.push_back(id);
        if (!j.finishing && j.pc < j.plan.size()) ready.push_back(id);
    }
    active_.swap(still);
    int K = 1;
    if (block_graphs_ && !ready.empty()) {
        int m = kBlockMax;
        for (int id : ready) m = std::min(m, device_run(*jobs_[id]));
        while (K * 2 <= m) K *= 2;  // a power of two: few distinct graphs
    }
    if (K >= 2) {
        if ((s = launch_block(K, ready))) return s;
    } else {
        t_fwd_->n = t_fwd_->tiles = 0;
        t_mid_->n = t_mid_->tiles = 0;
        t_adj_->n = t_adj_->tiles = 0;
        t_fus_->n = t_fus_->tiles = 0;
        for (int id : ready) {
            Job& j = *jobs_[id];
            if ((s = tick_action(j, j.plan[j.pc++]))) return s;
        }
        if ((s = launch_tick())) return s;
        ++ticks_;
    }
    if (active) *active = (int)active_.size();
    return FKADJ_OK;
}

int BatchEngine::device_run(const Job& j) const {
    int n = 0;
    for (size_t k = j.pc; k < j.plan.size() && n < kBlockMax; ++k, ++n) {
        const int kind = j.plan[k].kind;
        if (kind == Action::OBJ || kind == Action::FINISH) break;
    }
    return n;
}

// One tick: the four queues, packed into the next pinned ring slot and copied
// to the device queue in one stream-ordered copy (the previous tick's kernels
// are done with it by then); a slot is reused kQueueRing ticks later, after
// its copy's event.
fkadj_status BatchEngine::launch_tick() {
    const BatchInstance* inst = inst_dev_.as<BatchInstance>();
    const int nf = t_fwd_->n, nm = t_mid_->n, na = t_adj_->n, nu = t_fus_->n;
    if (nf + nm + na + nu > 0) {
        const int k = (int)(qcount_++ % kQueueRing);
        if (qev_[k]) BCK(cudaEventSynchronize(qev_[k]), "queue slot");
        else BCK(cudaEventCreateWithFlags(&qev_[k], cudaEventDisableTiming), "queue event");
        BatchItem* slot = qring_ + (size_t)k * 4 * kBatchMaxItems;
        std::copy(t_fwd_->item, t_fwd_->item + nf, slot);
        std::copy(t_mid_->item, t_mid_->item + nm, slot + nf);
        std::copy(t_adj_->item, t_adj_->item + na, slot + nf + nm);
        std::copy(t_fus_->item, t_fus_->item + nu, slot + nf + nm + na);
        BatchItem* dq = qdev_.as<BatchItem>();
        BCK(cudaMemcpyAsync(dq, slot, sizeof(BatchItem) * (size_t)(nf + nm + na + nu), cudaMemcpyHostToDevice, st_),
            "upload queue");
        BCK(cudaEventRecord(qev_[k], st_), "queue event");
        BCK(launch_batch_fwd(tiles_[0], inst, BatchQueue{dq, nf, t_fwd_->tiles}, st_), "batched forward");
        BCK(launch_batch_mid(tiles_[1], inst, BatchQueue{dq + nf, nm, t_mid_->tiles}, hw_, st_),
            "batched midpoint");
        BCK(launch_batch_adj(tiles_[2], inst, BatchQueue{dq + nf + nm, na, t_adj_->tiles}, st_),
            "batched adjoint");
        BCK(launch_batch_fused(tiles_[3], inst, BatchQueue{dq + nf + nm + na, nu, t_fus_->tiles}, hw_, st_),
            "batched fused adjoint");
    }
    launches_ += (nf > 0) + (nm > 0) + (na > 0) + (nu > 0);
    return FKADJ_OK;
}

// K ticks of the ready jobs (each takes its next K actions, all device work):
// the queues of tick t and kind k are planned into the staging slot, their
// header (n, tiles, first item) at [t][k]; one copy moves the slot to the
// device block, and a graph of K ticks x the kinds present replays the
// launches, each reading its header.  If this stream cannot be captured the
// same launches are issued directly.
fkadj_status BatchEngine::launch_block(int K, const std::vector<int>& ready) {
    const int r = (int)(bcount_++ % kBlockRing);
    if (bev_[r]) BCK(cudaEventSynchronize(bev_[r]), "block slot");
    else BCK(cudaEventCreateWithFlags(&bev_[r], cudaEventDisableTiming), "block event");
    char* slot = bring_ + (size_t)r * block_bytes();
    int* hdr = reinterpret_cast<int*>(slot);
    BatchItem* items = reinterpret_cast<BatchItem*>(slot + block_hdr_bytes());
    BatchTick* T[4] = {t_fwd_, t_mid_, t_adj_, t_fus_};
    int used = 0, mask = 0;
    fkadj_status s;
    for (int t = 0; t < K; ++t) {
        for (BatchTick* q : T) q->n = q->tiles = 0;
        for (int id : ready) {
            Job& j = *jobs_[id];
            if ((s = tick_action(j, j.plan[j.pc++]))) return s;
        }
        for (int k = 0; k < 4; ++k) {
            int* h = hdr + (t * 4 + k) * 4;
            h[0] = T[k]->n;
            h[1] = T[k]->tiles;
            h[2] = used;
            h[3] = 0;
            std::copy(T[k]->item, T[k]->item + T[k]->n, items + used);
            used += T[k]->n;
            if (T[k]->n > 0) mask |= 1 << k;
        }
    }
    BCK(cudaMemcpyAsync(bdev_.p, slot, block_hdr_bytes() + sizeof(BatchItem) * (size_t)used, cudaMemcpyHostToDevice,
                        st_),
        "upload block");
    BCK(cudaEventRecord(bev_[r], st_), "block event");
    const std::array<int, 6> key{K, mask, tiles_[0], tiles_[1], tiles_[2], tiles_[3]};
    const BatchInstance* inst = inst_dev_.as<BatchInstance>();
    const BatchItem* dbase = reinterpret_cast<const BatchItem*>(bdev_.as<char>() + block_hdr_bytes());
    const int* dhdr = bdev_.as<int>();
    auto issue = [&]() -> cudaError_t {
        cudaError_t e = cudaSuccess;
        for (int t = 0; t < K && e == cudaSuccess; ++t) {
            auto q = [&](int k) { return BatchQueue{dbase, 0, 0, dhdr + (t * 4 + k) * 4}; };
            if (!e && (mask & 1)) e = launch_batch_fwd(tiles_[0], inst, q(0), st_);
            if (!e && (mask & 2)) e = launch_batch_mid(tiles_[1], inst, q(1), hw_, st_);
            if (!e && (mask & 4)) e = launch_batch_adj(tiles_[2], inst, q(2), st_);
            if (!e && (mask & 8)) e = launch_batch_fused(tiles_[3], inst, q(3), hw_, st_);
        }
        return e;
    };
    cudaGraphExec_t gx = nullptr;
    for (auto& g : bgraphs_)
        if (g.first == key) gx = g.second;
    if (!gx) {
        cudaError_t e = cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            set_launch_pdl(false);
            e = issue();
            set_launch_pdl(true);
            cudaGraph_t graph = nullptr;
            const cudaError_t ec = cudaStreamEndCapture(st_, &graph);
            if (e == cudaSuccess) e = ec;
            if (e == cudaSuccess) e = cudaGraphInstantiate(&gx, graph, 0);
            if (graph) cudaGraphDestroy(graph);
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            gx = nullptr;
            block_graphs_ = false;
            BCK(issue(), "block launches");
            launches_ += (int64_t)K * __builtin_popcount(mask);
            ticks_ += K;
            return FKADJ_OK;
        }
        bgraphs_.push_back({key, gx});
    }
    BCK(cudaGraphLaunch(gx, st_), "block graph");
    launches_ += (int64_t)K * __builtin_popcount(mask);
    ticks_ += K;
    return FKADJ_OK;
}

fkadj_status BatchEngine::run_all() {
    int active = 1;
    fkadj_status s;
    while (active > 0) {
        if ((s = tick(&active))) return s;
        // only finishing jobs left: wait for the stream rather than spin
        bool all_finishing = true;
        for (int id : active_) all_finishing = all_finishing && jobs_[id]->finishing;
        if (active > 0 && all_finishing) BCK(cudaStreamSynchronize(st_), "synchronize");
    }
    return FKADJ_OK;
}

const Job* BatchEngine::job(int id) const {
    return (id >= 0 && id < (int)jobs_.size()) ? jobs_[id].get() : nullptr;
}

bool BatchEngine::job_done(int id) const {
    const Job* j = job(id);
    return j && j->done;
}

fkadj_status BatchEngine::job_result(int id, double* L0, double* LE, double* Lcost, double* gradE, int64_t n) {
    const Job* j = job(id);
    if (!j) {
        set_error("unknown job id");
        return FKADJ_ERR_ARG;
    }
    if (!j->done) {
        set_error("job not finished");
        return FKADJ_ERR_BUSY;
    }
    if (L0) *L0 = j->L0;
    if (LE) *LE = j->LE;
    if (Lcost) *Lcost = j->Lcost;
    if (gradE && j->want_grad) std::copy(j->gradE.begin(), j->gradE.begin() + std::min<int64_t>(n, j->gradE.size()), gradE);
    return j->status;
}

fkadj_status BatchEngine::release_job(int id) {
    if (id < 0 || id >= (int)jobs_.size() || !jobs_[id]) return FKADJ_OK;
    Job& j = *jobs_[id];
    if (!j.done) {
        set_error("job not finished");
        return FKADJ_ERR_BUSY;
    }
    if (j.ev) cudaEventDestroy(j.ev);
    if (j.h_out) give_pinned(j.h_out, j.h_cap);
    j.h_out = nullptr;
    jobs_[id].reset();
    return FKADJ_OK;
}

double* BatchEngine::take_pinned(size_t n, size_t* cap) {
    // smallest free buffer that holds n doubles
    int best = -1;
    for (int k = 0; k < (int)pinned_free_.size(); ++k)
        if (pinned_free_[k].first >= n && (best < 0 || pinned_free_[k].first < pinned_free_[best].first)) best = k;
    if (best >= 0) {
        double* p = pinned_free_[best].second;
        *cap = pinned_free_[best].first;
        pinned_free_.erase(pinned_free_.begin() + best);
        return p;
    }
    double* p = nullptr;
    if (cudaMallocHost(&p, n * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    *cap = n;
    return p;
}

void BatchEngine::give_pinned(double* p, size_t cap) {
    if (p) pinned_free_.push_back({cap, p});
}

}  // namespace fkadj

// ======================================================================= C ABI
struct fkadj_batch {
    fkadj::BatchEngine eng;
};

extern "C" {

fkadj_status fkadj_batch_create(fkadj_batch** out, const fkadj_options* opt) {
    if (!out) return FKADJ_ERR_ARG;
    *out = nullptr;
    auto* b = new (std::nothrow) fkadj_batch;
    if (!b) return FKADJ_ERR_NOMEM;
    fkadj_status s = b->eng.init(opt);
    if (s) {
        delete b;
        return s;
    }
    *out = b;
    return FKADJ_OK;
}

void fkadj_batch_destroy(fkadj_batch* b) { delete b; }

fkadj_status fkadj_batch_add_problem(fkadj_batch* b, const fkadj_params* p, double dt, int nt,
                                     const int* active_index, int nrows, int ncols, int n_num, const double* gh_num,
                                     const double* gamma, int64_t S_ncol, const int64_t* S_colptr,
                                     const int64_t* S_rowidx, const double* S_val, double alpha, int grad_mode,
                                     int ckpt_policy, int64_t ckpt_budget_bytes, int* problem_id) {
    if (!b || !p || !problem_id) {
        fkadj::set_error("null argument");
        return FKADJ_ERR_ARG;
    }
    return b->eng.add_problem(*p, dt, nt, active_index, nrows, ncols, n_num, gh_num, gamma, S_ncol, S_colptr,
                              S_rowidx, S_val, alpha, grad_mode, ckpt_policy, ckpt_budget_bytes, problem_id);
}

fkadj_status fkadj_batch_remove_problem(fkadj_batch* b, int problem_id) {
    if (!b) return FKADJ_ERR_ARG;
    return b->eng.remove_problem(problem_id);
}

fkadj_status fkadj_batch_submit(fkadj_batch* b, int problem_id, const double* Et, const double* y_ini,
                                int want_grad, int* job_id) {
    if (!b || !job_id) return FKADJ_ERR_ARG;
    return b->eng.submit(problem_id, Et, y_ini, want_grad != 0, job_id);
}

fkadj_status fkadj_batch_tick(fkadj_batch* b, int* active) {
    if (!b) return FKADJ_ERR_ARG;
    return b->eng.tick(active);
}

fkadj_status fkadj_batch_run(fkadj_batch* b) {
    if (!b) return FKADJ_ERR_ARG;
    return b->eng.run_all();
}

int fkadj_batch_job_done(const fkadj_batch* b, int job_id) { return b && b->eng.job_done(job_id) ? 1 : 0; }

fkadj_status fkadj_batch_result(fkadj_batch* b, int job_id, double* L0, double* LE, double* Lcost, double* gradE,
                                int64_t n_gradE) {
    if (!b) return FKADJ_ERR_ARG;
    return b->eng.job_result(job_id, L0, LE, Lcost, gradE, n_gradE);
}

fkadj_status fkadj_batch_release(fkadj_batch* b, int job_id) {
    if (!b) return FKADJ_ERR_ARG;
    return b->eng.release_job(job_id);
}

void fkadj_batch_stats(const fkadj_batch* b, int64_t out[3]) {
    if (!b || !out) return;
    out[0] = b->eng.launches();
    out[1] = b->eng.ticks();
    out[2] = b->eng.device_bytes();
}

}  // extern "C"
