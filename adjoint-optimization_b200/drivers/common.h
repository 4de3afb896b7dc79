// common.h -- shared pieces of the native drivers: MAT-file access with
// errors as exceptions, the inputs the reference's drivers load (grid, initial
// state, objective matrix), and the time stamps they put in file names.
#pragma once

#include <sys/time.h>
#include <unistd.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <ctime>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fkadj.h"
#include "../../include/fkadj_matio.h"

namespace fkadj_drivers {

inline void check(fkadj_status s, const std::string& what) {
    if (s != FKADJ_OK) throw std::runtime_error(what + ": " + fkadj_last_error());
}

class MatFile {
   public:
    explicit MatFile(const std::string& path) : path_(path) {
        check(fkadj_mat_open(path.c_str(), &m_), "reading " + path);
    }
    ~MatFile() { fkadj_mat_close(m_); }
    MatFile(const MatFile&) = delete;
    MatFile& operator=(const MatFile&) = delete;

    bool has(const std::string& name) const {
        for (int i = 0; i < fkadj_mat_count(m_); ++i)
            if (name == fkadj_mat_name(m_, i)) return true;
        return false;
    }
    int mx_class(const std::string& name) const {
        int c = 0;
        check(fkadj_mat_info(m_, name.c_str(), &c, nullptr, nullptr, 0, nullptr, nullptr, nullptr),
              path_);
        return c;
    }
    int64_t numel(const std::string& name) const {
        int64_t n = 0;
        check(fkadj_mat_info(m_, name.c_str(), nullptr, nullptr, nullptr, 0, &n, nullptr, nullptr),
              path_);
        return n;
    }
    std::vector<double> dbl(const std::string& name) const {
        std::vector<double> v((size_t)numel(name));
        check(fkadj_mat_read_double(m_, name.c_str(), v.data(), (int64_t)v.size()), path_);
        return v;
    }
    std::vector<int32_t> i32(const std::string& name) const {
        std::vector<int32_t> v((size_t)numel(name));
        check(fkadj_mat_read_int32(m_, name.c_str(), v.data(), (int64_t)v.size()), path_);
        return v;
    }
    double scalar(const std::string& name) const {
        std::vector<double> v = dbl(name);
        if (v.size() != 1) throw std::runtime_error(path_ + ": '" + name + "' is not a scalar");
        return v[0];
    }
    // Real sparse matrix as CSC with 64-bit indices.
    void sparse(const std::string& name, int64_t& nrows, int64_t& ncols, std::vector<int64_t>& colptr,
                std::vector<int64_t>& rowidx, std::vector<double>& val) const {
        int nd = 0, flags = 0;
        int64_t dims[2] = {0, 0}, nnz = 0;
        check(fkadj_mat_info(m_, name.c_str(), nullptr, &nd, dims, 2, nullptr, &nnz, &flags), path_);
        nrows = dims[0];
        ncols = dims[1];
        colptr.resize((size_t)ncols + 1);
        rowidx.resize((size_t)nnz);
        val.resize((size_t)nnz);
        check(fkadj_mat_read_sparse(m_, name.c_str(), colptr.data(), rowidx.data(), val.data()),
              path_);
    }

   private:
    std::string path_;
    fkadj_mat* m_ = nullptr;
};

class MatWriter {
   public:
    explicit MatWriter(const std::string& path, bool compress = true) {
        check(fkadj_matw_open(path.c_str(), compress ? 1 : 0, &w_), "creating " + path);
    }
    ~MatWriter() {
        if (w_) fkadj_matw_close(w_);
    }
    MatWriter(const MatWriter&) = delete;
    MatWriter& operator=(const MatWriter&) = delete;
    MatWriter& col(const char* name, const std::vector<double>& v) {
        check(fkadj_matw_dense(w_, name, FKADJ_MX_DOUBLE, (int64_t)v.size(), 1, v.data()), name);
        return *this;
    }
    MatWriter& row(const char* name, const std::vector<double>& v) {
        check(fkadj_matw_dense(w_, name, FKADJ_MX_DOUBLE, 1, (int64_t)v.size(), v.data()), name);
        return *this;
    }
    MatWriter& matrix(const char* name, int64_t rows, int64_t cols, const double* v) {
        check(fkadj_matw_dense(w_, name, FKADJ_MX_DOUBLE, rows, cols, v), name);
        return *this;
    }
    MatWriter& scalar(const char* name, double x) {
        check(fkadj_matw_dense(w_, name, FKADJ_MX_DOUBLE, 1, 1, &x), name);
        return *this;
    }
    MatWriter& str(const char* name, const std::string& s) {
        check(fkadj_matw_string(w_, name, s.c_str()), name);
        return *this;
    }
    void close() {
        fkadj_matw* w = w_;
        w_ = nullptr;
        check(fkadj_matw_close(w), "writing MAT file");
    }

   private:
    fkadj_matw* w_ = nullptr;
};

// The inputs both reference drivers load: active_index and ghost_lr from the
// grid file, and the compact initial state y0 = yf([bx;bx;bx]) with
// bx = active_index > 0 (simple_grad_desc.m:62-68, save_fk_forward_Et.m:88-104),
// or a stored y0 when the file has no yf.
struct Grid {
    std::vector<int32_t> active_index;
    std::vector<double> ghost_lr;
    int nrows = 0, ncols = 0, n_num = 0;
};

inline Grid load_grid(const std::string& path, int nrows, int ncols, bool require_int32) {
    MatFile f(path);
    Grid g;
    if (require_int32 && f.mx_class("active_index") != FKADJ_MX_INT32)
        throw std::runtime_error("Variable \"active_index\" must be of type int32");
    g.active_index = f.i32("active_index");
    g.ghost_lr = f.dbl("ghost_lr");
    const int64_t n = (int64_t)g.active_index.size();
    if (nrows <= 0 || ncols <= 0) {
        // the reference fixes 256 x 256 (simple_grad_desc.m:67-68); a square
        // grid is inferred from the length of active_index
        const int64_t side = (int64_t)std::llround(std::sqrt((double)n));
        if (side * side != n)
            throw std::runtime_error("active_index is not a square grid; set nrows and ncols");
        nrows = ncols = (int)side;
    }
    if ((int64_t)nrows * ncols != n)
        throw std::runtime_error("nrows*ncols does not match the length of active_index");
    g.nrows = nrows;
    g.ncols = ncols;
    for (int32_t a : g.active_index) g.n_num += a > 0;
    if ((int64_t)g.ghost_lr.size() != g.n_num)
        throw std::runtime_error("ghost_lr length does not match the active cells");
    return g;
}

inline std::vector<double> load_initial_state(const std::string& path, const Grid& g) {
    MatFile f(path);
    const size_t n = g.active_index.size();
    if (f.has("yf")) {
        const std::vector<double> yf = f.dbl("yf");
        if (yf.size() != 3 * n) throw std::runtime_error("yf must hold 3*nrows*ncols values");
        std::vector<double> y0;
        y0.reserve(3 * (size_t)g.n_num);
        for (int fld = 0; fld < 3; ++fld)
            for (size_t k = 0; k < n; ++k)
                if (g.active_index[k] > 0) y0.push_back(yf[fld * n + k]);
        return y0;
    }
    std::vector<double> y0 = f.dbl("y0");
    if (y0.size() != 3 * (size_t)g.n_num) throw std::runtime_error("y0 must hold 3*n_num values");
    return y0;
}

inline std::string hostname() {
    char h[256] = {0};
    if (gethostname(h, sizeof h - 1) != 0) throw std::runtime_error("Hostname not found");
    return h;
}

// str_clock_no_mu (src/cuda/str_clock_no_mu.m:1-15): 2024-nov-02-17-32-50.
inline std::string str_clock_no_mu() {
    static const char* month[] = {"jan", "feb", "mar", "apr", "may", "jun",
                                  "jul", "aug", "sep", "oct", "nov", "dec"};
    const time_t now = time(nullptr);
    struct tm t;
    localtime_r(&now, &t);
    char b[64];
    snprintf(b, sizeof b, "%04d-%s-%02d-%02d-%02d-%02d", t.tm_year + 1900, month[t.tm_mon],
             t.tm_mday, t.tm_hour, t.tm_min, t.tm_sec);
    return b;
}

inline double wall_seconds() {
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

}  // namespace fkadj_drivers
