// fkadj_simple_grad_desc -- native replacement of the reference's
// gradient-descent driver src/cuda/simple_grad_desc.m.
//
// Reads the same configuration file (default `infile_grad`, :22-35) and the
// same input files (seed pulse, initial state, grid, objective matrix,
// :52-70), takes ns gradient steps Et <- Et - ds*gradE (:78-107) with the
// problem resident on the GPU, records Lcost/L0/LE in Lcost_vec/L0_vec/LE_vec,
// and every nmod iterations writes simple_grad_desc_step_<time>_<jobid>_<i>.mat
// holding the variables the reference saves (:93-96), Et before its update.
//
// Keys beyond the reference's (all optional):
//   dt             time step in ms (the reference fixes 0.1, :45)
//   nrows, ncols   grid shape (the reference fixes 256 x 256, :67-68;
//                  default: inferred from a square active_index)
//   dx             grid spacing in cm of the FK parameter set (default 0.035)
//   grad_mode      'ref' (default, the reference's adjoint) or 'exact'
//   ckpt           'auto' (default), 'full', 'sqrt' or 'binomial'
//   ckpt_budget_gb trajectory-store budget (default: 60% of free memory)
//   line_search    'fixed' (default, the reference's step) or 'armijo': a
//                  backtracking search along -gradE whose trial steps
//                  ds*grow^k*beta^j run together as one batch of
//                  objective-only jobs (keys probes, beta, c1, grow)
//   device         CUDA device ordinal
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "common.h"
#include "infile.h"

using namespace fkadj_drivers;

namespace {

int ckpt_of(const std::string& s) {
    if (s == "auto") return FKADJ_CKPT_AUTO;
    if (s == "full") return FKADJ_CKPT_FULL;
    if (s == "sqrt") return FKADJ_CKPT_SQRT;
    if (s == "binomial") return FKADJ_CKPT_BINOMIAL;
    throw std::runtime_error("ckpt must be 'auto', 'full', 'sqrt' or 'binomial'");
}

int mode_of(const std::string& s) {
    if (s == "ref") return FKADJ_GRAD_REF;
    if (s == "exact") return FKADJ_GRAD_EXACT;
    throw std::runtime_error("grad_mode must be 'ref' or 'exact'");
}

struct Objective {
    int64_t nrows = 0, ncols = 0;
    std::vector<int64_t> colptr, rowidx;
    std::vector<double> val;
};

// Trial steps of one Armijo search, evaluated as one batch of objective-only
// jobs on `probes` resident copies of the problem.
class ProbeBatch {
   public:
    ProbeBatch(int probes, const fkadj_params& P, double dt, int nt, const Grid& g,
               const std::vector<double>& gamma, const Objective& S, double alpha,
               const fkadj_options& o, const std::vector<double>& y0)
        : y0_(y0) {
        check(fkadj_batch_create(&b_, &o), "batch");
        for (int k = 0; k < probes; ++k) {
            int id = -1;
            check(fkadj_batch_add_problem(b_, &P, dt, nt, g.active_index.data(), g.nrows, g.ncols,
                                          g.n_num, g.ghost_lr.data(), gamma.data(), S.ncols,
                                          S.colptr.data(), S.rowidx.data(), S.val.data(), alpha,
                                          o.grad_mode, o.ckpt_policy, o.ckpt_budget_bytes, &id),
                  "batch problem");
            ids_.push_back(id);
        }
    }
    ~ProbeBatch() { fkadj_batch_destroy(b_); }
    std::vector<double> lcost(const std::vector<std::vector<double>>& Es) {
        std::vector<int> jobs;
        for (size_t k = 0; k < Es.size(); ++k) {
            int j = -1;
            check(fkadj_batch_submit(b_, ids_[k], Es[k].data(), first_ ? y0_.data() : nullptr, 0, &j),
                  "probe");
            jobs.push_back(j);
        }
        first_ = false;
        check(fkadj_batch_run(b_), "probe batch");
        std::vector<double> out;
        for (int j : jobs) {
            double L0, LE, Lc;
            check(fkadj_batch_result(b_, j, &L0, &LE, &Lc, nullptr, 0), "probe result");
            check(fkadj_batch_release(b_, j), "probe release");
            out.push_back(Lc);
        }
        return out;
    }
    size_t size() const { return ids_.size(); }

   private:
    fkadj_batch* b_ = nullptr;
    std::vector<int> ids_;
    std::vector<double> y0_;
    bool first_ = true;
};

int run(const std::string& infile) {
    const std::string host = hostname();
    printf("hostname=\"%s\"\n", host.c_str());
    printf("****************start time= %s\n", str_clock_no_mu().c_str());
    const std::string program = "fkadj_simple_grad_desc";

    const Infile in(infile,
                    {"alpha", "ds", "ns", "final_time", "gamma", "nmod", "Et_seed_file", "icondfile",
                     "grid_file", "S_file", "mex_function", "in_path", "out_path", "jobid"},
                    {"dt", "nrows", "ncols", "dx", "grad_mode", "ckpt", "ckpt_budget_gb",
                     "line_search", "probes", "beta", "c1", "grow", "device"});
    printf("Parameters read from '%s' \n", infile.c_str());

    const double alpha = in.num("alpha"), ds = in.num("ds"), final_time = in.num("final_time");
    const long long ns = (long long)in.num("ns");
    const int nmod = (int)in.num("nmod");
    const std::vector<double> gamma = in.vec("gamma");
    if (gamma.size() != 3) throw std::runtime_error("gamma must have 3 entries");
    if (nmod < 1) throw std::runtime_error("nmod must be positive");
    const std::string Et_seed_file = in.str("Et_seed_file"), icondfile = in.str("icondfile");
    const std::string grid_file = in.str("grid_file"), S_file = in.str("S_file");
    const std::string mex_function = in.str("mex_function"), in_path = in.str("in_path");
    const std::string out_path = in.str("out_path"), jobid = in.str("jobid");
    const double dt = in.num_or("dt", 0.1);

    printf("alpha=%f\n", alpha);
    printf("ds=%f\n", ds);
    printf("ns=%f\n", (double)ns);
    printf("final_time=%f\n", final_time);
    printf("gamma=[%.2f, %.2f, %.2f]\n", gamma[0], gamma[1], gamma[2]);
    printf("Et_seed_file=%s\n", Et_seed_file.c_str());

    const long long nt = float_integer(final_time / dt);
    std::vector<double> Et = MatFile(in_path + Et_seed_file).dbl("Et");  // Et(:)
    if ((long long)Et.size() != nt + 1)
        throw std::runtime_error("Et has " + std::to_string(Et.size()) + " samples, nt+1 = " +
                                 std::to_string(nt + 1));
    const Grid g = load_grid(in_path + grid_file, (int)in.num_or("nrows", 0),
                             (int)in.num_or("ncols", 0), false);
    const std::vector<double> y0 = load_initial_state(in_path + icondfile, g);
    Objective S;
    MatFile(in_path + S_file).sparse("S", S.nrows, S.ncols, S.colptr, S.rowidx, S.val);

    fkadj_params P;
    fkadj_default_params(&P, in.num_or("dx", 0.035));
    fkadj_options o;
    fkadj_default_options(&o);
    o.grad_mode = mode_of(in.str_or("grad_mode", "ref"));
    o.ckpt_policy = ckpt_of(in.str_or("ckpt", "auto"));
    o.ckpt_budget_bytes = (int64_t)(in.num_or("ckpt_budget_gb", 0.0) * 1e9);
    o.device = (int)in.num_or("device", -1);
    const std::string search = in.str_or("line_search", "fixed");
    if (search != "fixed" && search != "armijo")
        throw std::runtime_error("line_search must be 'fixed' or 'armijo'");

    fkadj_problem* pb = nullptr;
    check(fkadj_problem_create(&pb, &P, dt, (int)nt, g.active_index.data(), g.nrows, g.ncols, g.n_num,
                               g.ghost_lr.data(), gamma.data(), S.ncols, S.colptr.data(),
                               S.rowidx.data(), S.val.data(), alpha, &o),
          "problem");
    std::unique_ptr<fkadj_problem, void (*)(fkadj_problem*)> hold(pb, fkadj_problem_destroy);
    std::unique_ptr<ProbeBatch> probes;
    if (search == "armijo")
        probes.reset(new ProbeBatch((int)in.num_or("probes", 6), P, dt, (int)nt, g, gamma, S, alpha, o,
                                    y0));
    const double beta = in.num_or("beta", 0.5), c1 = in.num_or("c1", 1e-4),
                 grow = in.num_or("grow", 2.0);
    double step = ds;

    const std::string time_str = str_clock_no_mu() + "_" + jobid;
    std::vector<double> Lcost_vec(nmod, 0.0), L0_vec(nmod, 0.0), LE_vec(nmod, 0.0);
    std::vector<double> gradE(nt + 1);
    for (long long i = 1; i <= ns; ++i) {
        puts("---------------- COMPUTING GRADIENT -------------");
        const double t0 = wall_seconds();
        double L0, LE, Lcost;
        check(fkadj_problem_grad(pb, Et.data(), i == 1 ? y0.data() : nullptr, &L0, &LE, &Lcost,
                                 gradE.data(), nullptr),
              "gradient");
        printf("time=%f\n", wall_seconds() - t0);

        const int ip = (int)((i - 1) % nmod);
        Lcost_vec[ip] = Lcost;
        L0_vec[ip] = L0;
        LE_vec[ip] = LE;

        if (i % nmod == 0) {  // Et is stored before it is updated
            const std::string outfile =
                "simple_grad_desc_step_" + time_str + "_" + std::to_string(i) + ".mat";
            puts(outfile.c_str());
            MatWriter w(out_path + outfile);
            w.scalar("alpha", alpha).scalar("dt", dt).scalar("final_time", final_time)
                .str("Et_seed_file", Et_seed_file).col("Et", Et).col("gradE", gradE)
                .scalar("Lcost", Lcost).scalar("ds", ds).col("Lcost_vec", Lcost_vec)
                .col("L0_vec", L0_vec).col("LE_vec", LE_vec).row("gamma", gamma)
                .str("program", program).str("hostname", host).scalar("nmod", nmod)
                .str("icondfile", icondfile).str("grid_file", grid_file).str("S_file", S_file)
                .str("mex_function", mex_function);
            w.close();
            printf("file \"%s%s\" written\n", out_path.c_str(), outfile.c_str());
        }

        if (!probes) {
            for (long long k = 0; k <= nt; ++k) Et[k] -= ds * gradE[k];
        } else {
            // slope of Lcost along d = -gradE: dt * gradE.d (gradE is
            // (1/dt) dLcost/dEt in the exact mode, its continuous-adjoint
            // approximation in the reference mode)
            double g2 = 0.0;
            for (double x : gradE) g2 += x * x;
            const double slope = -dt * g2;
            std::vector<double> steps;
            std::vector<std::vector<double>> Es;
            for (size_t k = 0; k < probes->size(); ++k) {
                steps.push_back(step * std::pow(beta, (double)k));
                Es.emplace_back(Et);
                for (long long m = 0; m <= nt; ++m) Es.back()[m] -= steps.back() * gradE[m];
            }
            const std::vector<double> Ls = probes->lcost(Es);
            size_t k = 0;
            while (k < Ls.size() && !(Ls[k] <= Lcost + c1 * steps[k] * slope)) ++k;
            if (k < Ls.size()) {
                Et = Es[k];
                printf("armijo: step %g accepted, Lcost %.12g -> %.12g\n", steps[k], Lcost, Ls[k]);
                step = k == 0 ? steps[0] * grow : steps[k];
            } else {
                printf("armijo: no step of %zu accepted (smallest %g)\n", Ls.size(), steps.back());
                step = steps.back() * beta;
            }
        }
        printf("********************* i_grad = %lld of %lld\n", i, ns);
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        return run(argc > 1 ? argv[1] : "infile_grad");
    } catch (const std::exception& e) {
        fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
}
