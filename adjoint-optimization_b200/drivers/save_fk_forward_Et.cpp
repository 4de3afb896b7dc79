// fkadj_save_fk_forward_Et -- native replacement of the reference's forward
// driver src/cuda/save_fk_forward_Et.m.
//
// Reads the same configuration file (default `infile_forward`, :24-41), the
// pulse file (alpha when present, dt, final_time, Et; or Et = 0 over
// final_time at dt = 0.1 when Et_file is empty, :48-71), the grid file
// (active_index must be int32, :77-85) and the initial state (yf, else y0,
// :88-95); runs the forward sweep with snapshots every nstep steps; writes
// ys, yf, nrows, ncols, icondfile, dt, nstep, final_time, grid_file,
// param_str, Et_file, program, mex_function and hostname to out_path/outfile,
// outfile defaulting to outfile_prefix + Et_file (:100-117).
//
// Keys beyond the reference's (optional): nrows, ncols (the reference fixes
// 256 x 256, :97-98), dx (default 0.035) and device.
#include <cstdio>
#include <string>
#include <vector>

#include "common.h"
#include "infile.h"

using namespace fkadj_drivers;

namespace {

// compute_ns of src/cuda/fk_forward_Et_param_mex.cpp:7-25: the final state is
// not stored in ys when nt/nstep is an integer.
int compute_ns(double nt, double nstep) {
    const double r = nt / nstep, rn = std::round(r);
    if (std::fabs(r - rn) < 5e-16 * r) {
        printf("nt/nstep is an integer\n");
        printf("ns=nt/nstep-1=%d\n", (int)rn - 1);
        return (int)rn - 1;
    }
    printf("nt/nstep is not an integer\n");
    printf("ns = floor(nt/nstep)=%d\n", (int)std::floor(r));
    return (int)std::floor(r);
}

int run(const std::string& infile) {
    const std::string host = hostname();
    printf("hostname=\"%s\"\n", host.c_str());
    const std::string program = "fkadj_save_fk_forward_Et";

    const Infile in(infile,
                    {"Et_file", "final_time", "nstep", "icondfile", "outfile", "outfile_prefix",
                     "mex_function", "grid_file", "in_path", "out_path"},
                    {"nrows", "ncols", "dx", "device"});
    printf("Parameters read from '%s' \n", infile.c_str());
    const std::string Et_file = in.str("Et_file"), icondfile = in.str("icondfile");
    const std::string grid_file = in.str("grid_file"), in_path = in.str("in_path");
    const std::string out_path = in.str("out_path"), mex_function = in.str("mex_function");
    std::string outfile = in.str("outfile");
    const std::string outfile_prefix = in.str("outfile_prefix");
    const double nstep = in.num("nstep");
    double final_time = in.num("final_time"), dt;
    std::vector<double> Et;
    long long nt;
    if (!Et_file.empty()) {
        MatFile f(in_path + Et_file);
        if (f.has("alpha")) printf("alpha=%g\n", f.scalar("alpha"));
        else printf("No alpha found in Et_file \"%s\"\n", Et_file.c_str());
        dt = f.scalar("dt");
        final_time = f.scalar("final_time");
        Et = f.dbl("Et");
        nt = float_integer(final_time / dt);
    } else {
        printf("Et_file string is empty, will set Et to zero\n");
        dt = 0.1;
        nt = float_integer(final_time / dt);
        Et.assign((size_t)nt + 1, 0.0);
    }
    if ((long long)Et.size() != nt + 1)
        throw std::runtime_error("Et has " + std::to_string(Et.size()) + " samples, nt+1 = " +
                                 std::to_string(nt + 1));

    const Grid g = load_grid(in_path + grid_file, (int)in.num_or("nrows", 0),
                             (int)in.num_or("ncols", 0), true);
    const std::vector<double> y0 = load_initial_state(in_path + icondfile, g);

    if (outfile.empty()) {
        if (Et_file.empty()) throw std::runtime_error("Et_file is empty. Cannot generate outfile");
        if (outfile_prefix.empty())
            throw std::runtime_error("outfile_prefix is empty. Cannot generate outfile");
        outfile = outfile_prefix + Et_file;
    }

    fkadj_params P;
    fkadj_default_params(&P, in.num_or("dx", 0.035));
    fkadj_options o;
    fkadj_default_options(&o);
    o.device = (int)in.num_or("device", -1);
    const int ns = compute_ns((double)nt, nstep);
    const size_t n3 = 3 * g.active_index.size();
    std::vector<double> ys(n3 * (size_t)std::max(ns, 0)), yf(n3);
    const double t0 = wall_seconds();
    check(fkadj_forward(&P, dt, Et.data(), (int)nt, y0.data(), g.active_index.data(), g.nrows,
                        g.ncols, g.n_num, g.ghost_lr.data(), (int)nstep, ns,
                        ns > 0 ? ys.data() : nullptr, yf.data(), &o),
          "forward");
    printf("forward: %.3f s\n", wall_seconds() - t0);
    const std::string param_str = fkadj_param_string(&P);

    MatWriter w(out_path + outfile);
    w.matrix("ys", (int64_t)n3, ns > 0 ? ns : 0, ys.data()).col("yf", yf)
        .scalar("nrows", g.nrows).scalar("ncols", g.ncols).str("icondfile", icondfile)
        .scalar("dt", dt).scalar("nstep", nstep).scalar("final_time", final_time)
        .str("grid_file", grid_file).str("param_str", param_str).str("Et_file", Et_file)
        .str("program", program).str("mex_function", mex_function).str("hostname", host);
    w.close();
    printf("Saved file \"%s%s\"\n", out_path.c_str(), outfile.c_str());
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        return run(argc > 1 ? argv[1] : "infile_forward");
    } catch (const std::exception& e) {
        fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
}
