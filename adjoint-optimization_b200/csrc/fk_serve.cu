// fk_serve.cu -- continuous-batching request server.
//
// Clients submit objective or objective+gradient requests from any thread; a
// worker thread owns the GPU and the BatchEngine.  Between ticks it admits
// queued requests in arrival order while their estimated device footprint fits
// the HBM budget and fewer than the engine's maximum jobs run; an admitted
// request's problem (geometry, objective, trajectory store) is created on the
// device and its job joins the next tick, so requests that arrive while others
// run share every launch with them.  Finished jobs hand their results back and
// free their memory.  Waits on the client side are bounded.  The reference has
// no serving path (one synchronous MATLAB call per gradient).
//
// Two ways to run the admitted requests (FKADJ_SERVE_MODE):
//   streams (default)  a pool of worker threads (FKADJ_SERVE_STREAMS, 4), each
//       taking the next admitted request and running it through the
//       single-instance path on its own stream: the requests' kernels overlap
//       on the device wherever SMs are free, and each request gets the
//       single-instance kernels (one-wave tiles, kept f, bulk tile copies).
//   ticks  one worker thread ticking a BatchEngine: every running request's
//       next step joins one persistent launch per kernel kind.
// Admission is the same: arrival order, while the estimated device footprint
// fits the budget.  Measured on B200 the tick engine served a stream of
// 128^2..512^2 requests slower than plain one-at-a-time solves, the stream
// workers faster.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>

#include "fk_batch.h"

namespace fkadj {

struct Request {
    int64_t id = 0;
    fkadj_params p{};
    double dt = 0, alpha = 0;
    int nt = 0, nrows = 0, ncols = 0, n_num = 0;
    std::vector<int> ai;
    std::vector<double> gh, gamma, Sv, Et, y0;
    std::vector<int64_t> Jc, Ir;
    bool want_grad = true;
    int64_t est = 0;
    // results
    int state = 0;  // 0 queued, 1 running, 2 done, 3 failed
    fkadj_status status = FKADJ_OK;
    std::string err;
    double L0 = 0, LE = 0, Lcost = 0;
    std::vector<double> gradE;
    double t_submit = 0, t_admit = 0, t_done = 0;
    int prob = -1, job = -1;
};

class Server {
public:
    ~Server() { stop(); }
    fkadj_status start(const fkadj_options* opt, int64_t budget);
    void stop();
    fkadj_status submit(std::unique_ptr<Request> r, int64_t* id);
    int poll(int64_t id);
    fkadj_status wait(int64_t id, double timeout_s);
    fkadj_status result(int64_t id, double* L0, double* LE, double* Lcost, double* gradE, int64_t n, double* lat);
    void stats(int64_t out[6]);

private:
    void loop();
    void worker();
    fkadj_status admit(Request& r);
    fkadj_status run_alone(Request& r);
    bool streams_ = true;
    int nworkers_ = 4;
    std::vector<std::thread> workers_;
    fkadj_options opt_{};
    int device_ = 0;
    int64_t budget_ = 0, used_ = 0;
    std::unique_ptr<BatchEngine> eng_;
    std::thread th_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    std::deque<int64_t> queue_;
    std::map<int64_t, std::unique_ptr<Request>> reqs_;
    std::vector<int64_t> running_;
    std::atomic<bool> stop_{false};
    int64_t next_id_ = 1, completed_ = 0, failed_ = 0, peak_running_ = 0;
    fkadj_status init_status_ = FKADJ_OK;
    bool started_ = false;
};

fkadj_status Server::start(const fkadj_options* opt, int64_t budget) {
    fkadj_default_options(&opt_);
    if (opt) opt_ = *opt;
    if (opt_.device >= 0) {
        device_ = opt_.device;
    } else if (cudaGetDevice(&device_) != cudaSuccess) {
        set_error("no CUDA device");
        return FKADJ_ERR_NODEVICE;
    }
    if (budget <= 0) {
        size_t fr = 0, tot = 0;
        cudaSetDevice(device_);
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            set_error("cudaMemGetInfo failed");
            return FKADJ_ERR_CUDA;
        }
        budget = (int64_t)(0.8 * (double)fr);
    }
    budget_ = budget;
    if (const char* m = getenv("FKADJ_SERVE_MODE")) streams_ = std::strcmp(m, "ticks") != 0;
    if (const char* w = getenv("FKADJ_SERVE_STREAMS")) nworkers_ = std::max(1, std::min(64, std::atoi(w)));
    if (streams_) {
        for (int k = 0; k < nworkers_; ++k) workers_.emplace_back([this] { worker(); });
        return FKADJ_OK;
    }
    std::unique_lock<std::mutex> lk(mu_);
    th_ = std::thread([this] { loop(); });
    cv_.wait(lk, [this] { return started_; });
    return init_status_;
}

void Server::stop() {
    stop_ = true;
    cv_.notify_all();
    for (auto& w : workers_)
        if (w.joinable()) w.join();
    workers_.clear();
    if (th_.joinable()) th_.join();
}

// One request through the single-instance path on the worker's own problem
// and stream: device memory from the per-device stream-ordered pool (no
// device-wide synchronisation when it is freed), tiles from the autotuner's
// cache for the grid shape.
fkadj_status Server::run_alone(Request& r) {
    auto pb = std::make_unique<Problem>();
    pb->set_oneshot(oneshot_pool(&opt_));
    fkadj_options o = opt_;
    o.stream = nullptr;
    o.device = device_;
    o.ckpt_policy = opt_.ckpt_policy == FKADJ_CKPT_FULL ? FKADJ_CKPT_FULL : FKADJ_CKPT_SQRT;
    o.ckpt_budget_bytes = budget_;
    fkadj_status s = pb->init(r.p, r.dt, r.nt, r.ai.data(), r.nrows, r.ncols, r.n_num, r.gh.data(), r.gamma.data(),
                              r.n_num, r.Jc.data(), r.Ir.data(), r.Sv.data(), r.alpha, &o, true);
    if (s) return s;
    if (r.want_grad) {
        std::vector<double> g(r.nt + 1);
        s = pb->grad(r.Et.data(), r.y0.data(), &r.L0, &r.LE, &r.Lcost, g.data(), nullptr);
        r.gradE.swap(g);
    } else {
        s = pb->objective(r.Et.data(), r.y0.data(), &r.L0, &r.LE, &r.Lcost, nullptr);
    }
    return s;
}

void Server::worker() {
    if (cudaSetDevice(device_) != cudaSuccess) return;
    while (true) {
        int64_t id = 0;
        Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu_);
            // the front request, once its footprint fits beside the running ones
            cv_.wait(lk, [this] {
                if (stop_) return true;
                if (queue_.empty()) return false;
                const Request& f = *reqs_[queue_.front()];
                return running_.empty() || used_ + f.est <= budget_;
            });
            if (stop_ && queue_.empty()) return;
            if (queue_.empty()) continue;
            id = queue_.front();
            queue_.pop_front();
            r = reqs_[id].get();
            r->state = 1;
            r->t_admit = host_seconds();
            used_ += r->est;
            running_.push_back(id);
            peak_running_ = std::max<int64_t>(peak_running_, (int64_t)running_.size());
        }
        const fkadj_status s = run_alone(*r);
        {
            std::lock_guard<std::mutex> lk(mu_);
            r->status = s;
            r->state = (s == FKADJ_OK || s == FKADJ_ERR_NUMERIC) ? 2 : 3;
            if (r->state == 3) {
                r->err = fkadj_last_error();
                ++failed_;
            } else {
                ++completed_;
            }
            r->t_done = host_seconds();
            used_ -= r->est;
            running_.erase(std::find(running_.begin(), running_.end(), id));
        }
        done_cv_.notify_all();
        cv_.notify_all();  // memory freed: the next request may fit now
    }
}

fkadj_status Server::submit(std::unique_ptr<Request> r, int64_t* id) {
    r->t_submit = host_seconds();
    r->est = Problem::estimate_bytes(r->nrows, r->ncols, r->nt, r->n_num, (int64_t)r->Sv.size(), opt_.grad_mode,
                                     opt_.ckpt_policy == FKADJ_CKPT_FULL ? FKADJ_CKPT_FULL : FKADJ_CKPT_SQRT,
                                     r->want_grad);
    if (r->est > budget_) {
        set_error("request does not fit the HBM budget even alone");
        return FKADJ_ERR_NOMEM;
    }
    {
        std::lock_guard<std::mutex> lk(mu_);
        r->id = next_id_++;
        *id = r->id;
        queue_.push_back(r->id);
        reqs_[r->id] = std::move(r);
    }
    cv_.notify_all();
    return FKADJ_OK;
}

fkadj_status Server::admit(Request& r) {
    int pid = -1;
    const int policy = opt_.ckpt_policy == FKADJ_CKPT_FULL ? FKADJ_CKPT_FULL : FKADJ_CKPT_SQRT;
    fkadj_status s = eng_->add_problem(r.p, r.dt, r.nt, r.ai.data(), r.nrows, r.ncols, r.n_num, r.gh.data(),
                                       r.gamma.data(), r.n_num, r.Jc.data(), r.Ir.data(), r.Sv.data(), r.alpha,
                                       opt_.grad_mode, policy, budget_, &pid);
    if (s) return s;
    int job = -1;
    s = eng_->submit(pid, r.Et.data(), r.y0.data(), r.want_grad, &job);
    if (s) {
        eng_->remove_problem(pid);
        return s;
    }
    r.prob = pid;
    r.job = job;
    r.t_admit = host_seconds();
    return FKADJ_OK;
}

void Server::loop() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (cudaSetDevice(device_) != cudaSuccess) {
            init_status_ = FKADJ_ERR_NODEVICE;
        } else {
            eng_ = std::make_unique<BatchEngine>();
            fkadj_options o = opt_;
            o.stream = nullptr;
            init_status_ = eng_->init(&o);
        }
        started_ = true;
    }
    cv_.notify_all();
    if (init_status_) return;
    while (true) {
        // admissions, in arrival order
        {
            std::unique_lock<std::mutex> lk(mu_);
            if (running_.empty() && queue_.empty()) {
                if (stop_) break;
                cv_.wait_for(lk, std::chrono::milliseconds(2));
                continue;
            }
            while (!queue_.empty() && (int)running_.size() < kBatchMaxItems) {
                Request& r = *reqs_[queue_.front()];
                if (used_ + r.est > budget_ && !running_.empty()) break;
                lk.unlock();
                fkadj_status s = admit(r);
                lk.lock();
                queue_.pop_front();
                if (s) {
                    r.state = 3;
                    r.status = s;
                    r.err = fkadj_last_error();
                    r.t_done = host_seconds();
                    ++failed_;
                    done_cv_.notify_all();
                    continue;
                }
                r.state = 1;
                used_ += r.est;
                running_.push_back(r.id);
                peak_running_ = std::max<int64_t>(peak_running_, (int64_t)running_.size());
            }
        }
        int active = 0;
        fkadj_status s = eng_->tick(&active);
        // completions
        std::vector<int64_t> finished;
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (int64_t id : running_) {
                Request& r = *reqs_[id];
                if (s || eng_->job_done(r.job)) finished.push_back(id);
            }
        }
        for (int64_t id : finished) {
            Request* r;
            {
                std::lock_guard<std::mutex> lk(mu_);
                r = reqs_[id].get();
            }
            std::vector<double> g(r->want_grad ? r->nt + 1 : 0);
            fkadj_status rs = s ? s : eng_->job_result(r->job, &r->L0, &r->LE, &r->Lcost, g.data(), (int64_t)g.size());
            if (!s) {
                eng_->release_job(r->job);
                eng_->remove_problem(r->prob);
            }
            std::lock_guard<std::mutex> lk(mu_);
            r->gradE.swap(g);
            r->status = rs;
            r->state = (rs == FKADJ_OK || rs == FKADJ_ERR_NUMERIC) ? 2 : 3;
            if (r->state == 3) {
                r->err = fkadj_last_error();
                ++failed_;
            } else {
                ++completed_;
            }
            r->t_done = host_seconds();
            used_ -= r->est;
            running_.erase(std::find(running_.begin(), running_.end(), id));
            done_cv_.notify_all();
        }
        if (s) {  // engine failure: fail everything queued too
            std::lock_guard<std::mutex> lk(mu_);
            for (int64_t id : queue_) {
                reqs_[id]->state = 3;
                reqs_[id]->status = s;
                reqs_[id]->t_done = host_seconds();
            }
            queue_.clear();
            done_cv_.notify_all();
            break;
        }
        // only jobs waiting for their final copy: let the GPU drain briefly
        if (active > 0) {
            bool all_fin = true;
            for (int64_t id : running_) {
                const Job* j = eng_->job(reqs_[id]->job);
                all_fin = all_fin && j && j->finishing;
            }
            if (all_fin) cudaStreamSynchronize(eng_->stream());
        }
    }
    eng_.reset();
}

int Server::poll(int64_t id) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return -1;
    return it->second->state == 2 ? 1 : (it->second->state == 3 ? -2 : 0);
}

fkadj_status Server::wait(int64_t id, double timeout_s) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) {
        set_error("unknown request");
        return FKADJ_ERR_ARG;
    }
    Request* r = it->second.get();
    const bool ok = done_cv_.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                      [r] { return r->state >= 2; });
    if (!ok) {
        set_error("timed out waiting for the request");
        return FKADJ_ERR_TIMEOUT;
    }
    if (r->state == 2) return FKADJ_OK;
    // the failure's message belongs to the thread that ran the request
    set_error(r->err.empty() ? "request failed" : r->err);
    return r->status;
}

fkadj_status Server::result(int64_t id, double* L0, double* LE, double* Lcost, double* gradE, int64_t n,
                            double* lat) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) {
        set_error("unknown request");
        return FKADJ_ERR_ARG;
    }
    Request& r = *it->second;
    if (r.state < 2) {
        set_error("request not finished");
        return FKADJ_ERR_BUSY;
    }
    if (r.state == 3) {
        set_error(r.err.empty() ? "request failed" : r.err);
        return r.status;
    }
    if (L0) *L0 = r.L0;
    if (LE) *LE = r.LE;
    if (Lcost) *Lcost = r.Lcost;
    if (gradE) std::copy(r.gradE.begin(), r.gradE.begin() + std::min<int64_t>(n, (int64_t)r.gradE.size()), gradE);
    if (lat) {
        lat[0] = r.t_done - r.t_submit;  // latency
        lat[1] = r.t_admit - r.t_submit;  // queueing
    }
    fkadj_status st = r.status;
    reqs_.erase(it);
    return st;
}

void Server::stats(int64_t out[6]) {
    std::lock_guard<std::mutex> lk(mu_);
    out[0] = completed_;
    out[1] = failed_;
    out[2] = (int64_t)queue_.size();
    out[3] = (int64_t)running_.size();
    out[4] = peak_running_;
    out[5] = used_;
}

}  // namespace fkadj

// ======================================================================= C ABI
struct fkadj_server {
    fkadj::Server srv;
};

extern "C" {

fkadj_status fkadj_server_create(fkadj_server** out, const fkadj_options* opt, int64_t hbm_budget_bytes) {
    if (!out) return FKADJ_ERR_ARG;
    *out = nullptr;
    auto* s = new (std::nothrow) fkadj_server;
    if (!s) return FKADJ_ERR_NOMEM;
    fkadj_status st = s->srv.start(opt, hbm_budget_bytes);
    if (st) {
        delete s;
        return st;
    }
    *out = s;
    return FKADJ_OK;
}

void fkadj_server_destroy(fkadj_server* s) { delete s; }

fkadj_status fkadj_server_submit(fkadj_server* s, const fkadj_params* p, double dt, int nt, const int* active_index,
                                 int nrows, int ncols, int n_num, const double* gh_num, const double* gamma,
                                 int64_t S_ncol, const int64_t* S_colptr, const int64_t* S_rowidx,
                                 const double* S_val, double alpha, const double* Et, const double* y_ini,
                                 int want_grad, int64_t* request_id) {
    if (!s || !p || !active_index || !gh_num || !gamma || !S_colptr || !S_rowidx || !S_val || !Et || !y_ini ||
        !request_id || nt < 3 || nrows < 2 || ncols < 2 || n_num < 1 || S_ncol != n_num) {
        fkadj::set_error("invalid server request");
        return FKADJ_ERR_ARG;
    }
    auto r = std::make_unique<fkadj::Request>();
    r->p = *p;
    r->dt = dt;
    r->nt = nt;
    r->nrows = nrows;
    r->ncols = ncols;
    r->n_num = n_num;
    r->alpha = alpha;
    r->ai.assign(active_index, active_index + (size_t)nrows * ncols);
    r->gh.assign(gh_num, gh_num + n_num);
    r->gamma.assign(gamma, gamma + 3);
    r->Jc.assign(S_colptr, S_colptr + n_num + 1);
    r->Ir.assign(S_rowidx, S_rowidx + S_colptr[n_num]);
    r->Sv.assign(S_val, S_val + S_colptr[n_num]);
    r->Et.assign(Et, Et + nt + 1);
    r->y0.assign(y_ini, y_ini + (size_t)3 * n_num);
    r->want_grad = want_grad != 0;
    return s->srv.submit(std::move(r), request_id);
}

int fkadj_server_poll(fkadj_server* s, int64_t request_id) { return s ? s->srv.poll(request_id) : -1; }

fkadj_status fkadj_server_wait(fkadj_server* s, int64_t request_id, double timeout_s) {
    if (!s) return FKADJ_ERR_ARG;
    return s->srv.wait(request_id, timeout_s);
}

fkadj_status fkadj_server_result(fkadj_server* s, int64_t request_id, double* L0, double* LE, double* Lcost,
                                 double* gradE, int64_t n_gradE, double latency_s[2]) {
    if (!s) return FKADJ_ERR_ARG;
    return s->srv.result(request_id, L0, LE, Lcost, gradE, n_gradE, latency_s);
}

void fkadj_server_stats(fkadj_server* s, int64_t out[6]) {
    if (s && out) s->srv.stats(out);
}

}  // extern "C"
