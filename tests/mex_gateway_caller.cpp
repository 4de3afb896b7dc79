// Test program (built by tests/test_gpu_mex_shim.py): a caller shaped like the
// reference's gradient gateway (src/cuda/fk_grad_Et_param_mex.cpp:26-38 unpacks
// the arguments, :69-79 allocates the outputs and calls fk_grad_Et_comp),
// compiled against the MEX-API stand-in and include/fkadj_mex_compat.h, so the
// call goes through the shim's reference name and signature: the objective
// matrix arrives as a CSC mxArray with mwIndex (size_t) row indices and column
// pointers, and the spacing is the shim's default FKADJ_MEX_DX.
//
// Usage: mex_gateway_caller <dir>.  Reads from <dir> the raw little-endian
// files written by the test:
//   scalars.f64  dt, nt, nrows, ncols, n_num, alpha, nnz   (7 doubles)
//   Et.f64 (nt+1), y0.f64 (3 n_num), active_index.i32 (nrows*ncols),
//   ghost.f64 (n_num), gamma.f64 (3), S_jc.u64 (n_num+1), S_ir.u64 (nnz),
//   S_pr.f64 (nnz)
// and writes out.f64 = [status, Lcost, L0, LE, gradE (nt+1)] and param.txt.
#include <cstdio>
#include <string>
#include <vector>

#include "matrix.h"
#include "fkadj_mex_compat.h"

template <class T>
static bool load(const std::string& path, std::vector<T>& v, size_t n) {
    v.resize(n);
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    const size_t got = std::fread(v.data(), sizeof(T), n, f);
    std::fclose(f);
    return got == n;
}

int main(int argc, char** argv) {
    if (argc != 2) return 2;
    const std::string d = std::string(argv[1]) + "/";
    std::vector<double> sc;
    if (!load(d + "scalars.f64", sc, 7)) return 3;
    const double dt = sc[0], alpha = sc[5];
    const int nt = (int)sc[1], nrows = (int)sc[2], ncols = (int)sc[3], n_num = (int)sc[4];
    const size_t nnz = (size_t)sc[6];
    std::vector<double> Et, y0, ghost, gamma, pr;
    std::vector<int> ai;
    std::vector<mwIndex> jc, ir;
    if (!load(d + "Et.f64", Et, nt + 1) || !load(d + "y0.f64", y0, 3 * (size_t)n_num) ||
        !load(d + "active_index.i32", ai, (size_t)nrows * ncols) || !load(d + "ghost.f64", ghost, n_num) ||
        !load(d + "gamma.f64", gamma, 3) || !load(d + "S_jc.u64", jc, n_num + 1) || !load(d + "S_ir.u64", ir, nnz) ||
        !load(d + "S_pr.f64", pr, nnz))
        return 4;
    // the sparse S the gateway receives as prhs[9]
    mxArray S = {};
    S.m = (size_t)n_num;
    S.n = (size_t)n_num;
    S.pr = pr.data();
    S.ir = ir.data();
    S.jc = jc.data();
    S.owns = 0;
    // outputs allocated by the caller, as the gateway does (fk_grad_Et_param_mex.cpp:69-79)
    mxArray* gradE = mxCreateDoubleMatrix(nt + 1, 1, mxREAL);
    double L0 = 0, LE = 0, Lcost = 0;
    char* param_str = nullptr;
    const int rc = fk_grad_Et_comp(dt, Et.data(), nt, y0.data(), ai.data(), nrows, ncols, n_num, ghost.data(),
                                   gamma.data(), &S, alpha, &L0, &LE, &Lcost, mxGetPr(gradE), &param_str);
    std::vector<double> out = {(double)rc, Lcost, L0, LE};
    out.insert(out.end(), mxGetPr(gradE), mxGetPr(gradE) + nt + 1);
    FILE* f = std::fopen((d + "out.f64").c_str(), "wb");
    if (!f) return 5;
    std::fwrite(out.data(), sizeof(double), out.size(), f);
    std::fclose(f);
    if (param_str) {
        FILE* p = std::fopen((d + "param.txt").c_str(), "w");
        if (p) {
            std::fputs(param_str, p);
            std::fclose(p);
        }
        mxFree(param_str);
    }
    mxDestroyArray(gradE);
    return rc == 0 ? 0 : 1;
}
