// fk_matio.cpp -- MAT-file level-5 reader and writer (include/fkadj_matio.h).
//
// Written from the published layout of the level-5 format: a 128-byte header
// (text, subsystem offset, version 0x0100, endian mark "IM"), then data
// elements, each an 8-byte tag (type, byte count) or a 4-byte "small" tag
// packing both into one word, with payloads padded to 8 bytes.  A variable is
// an miMATRIX element holding array flags, dimensions, name and the real (and
// imaginary) parts, or ir/jc/pr for sparse; miCOMPRESSED wraps one element in
// a zlib stream.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include <zlib.h>

#include "../../include/fkadj_matio.h"
#include "fk_engine.h"

namespace {

using fkadj::set_error;

enum MiType {
    miINT8 = 1, miUINT8 = 2, miINT16 = 3, miUINT16 = 4, miINT32 = 5, miUINT32 = 6,
    miSINGLE = 7, miDOUBLE = 9, miINT64 = 12, miUINT64 = 13, miMATRIX = 14,
    miCOMPRESSED = 15, miUTF8 = 16, miUTF16 = 17, miUTF32 = 18
};

int mi_size(uint32_t t) {
    switch (t) {
        case miINT8: case miUINT8: case miUTF8: return 1;
        case miINT16: case miUINT16: case miUTF16: return 2;
        case miINT32: case miUINT32: case miSINGLE: case miUTF32: return 4;
        case miDOUBLE: case miINT64: case miUINT64: return 8;
        default: return 0;
    }
}

// One numeric payload as stored: its type and raw bytes.
struct Part {
    uint32_t type = 0;
    std::vector<uint8_t> bytes;
    int64_t count() const { return mi_size(type) ? (int64_t)bytes.size() / mi_size(type) : 0; }
    double at(int64_t i) const {
        const uint8_t* p = bytes.data() + i * mi_size(type);
        switch (type) {
            case miINT8: return (double)*(const int8_t*)p;
            case miUINT8: case miUTF8: return (double)*p;
            case miINT16: { int16_t v; memcpy(&v, p, 2); return v; }
            case miUINT16: case miUTF16: { uint16_t v; memcpy(&v, p, 2); return v; }
            case miINT32: { int32_t v; memcpy(&v, p, 4); return v; }
            case miUINT32: case miUTF32: { uint32_t v; memcpy(&v, p, 4); return v; }
            case miSINGLE: { float v; memcpy(&v, p, 4); return v; }
            case miDOUBLE: { double v; memcpy(&v, p, 8); return v; }
            case miINT64: { int64_t v; memcpy(&v, p, 8); return (double)v; }
            case miUINT64: { uint64_t v; memcpy(&v, p, 8); return (double)v; }
            default: return std::numeric_limits<double>::quiet_NaN();
        }
    }
    // exact integer value (for indices and int32 reads); false when the value
    // is not an integer or does not fit in 64 bits
    bool int_at(int64_t i, int64_t& out) const {
        const uint8_t* p = bytes.data() + i * mi_size(type);
        if (type == miINT64) { memcpy(&out, p, 8); return true; }
        if (type == miUINT64) {
            uint64_t v; memcpy(&v, p, 8);
            if (v > (uint64_t)INT64_MAX) return false;
            out = (int64_t)v; return true;
        }
        const double d = at(i);
        if (!(d == std::floor(d)) || std::fabs(d) > 9.0e15) return false;
        out = (int64_t)d;
        return true;
    }
};

struct Var {
    std::string name;
    int cls = 0;
    bool complex = false, logical = false, readable = false;
    std::vector<int64_t> dims;
    Part re, im;      // dense data, or pr / pi for sparse
    Part ir, jc;      // sparse indices
    int64_t numel() const {
        int64_t n = 1;
        for (int64_t d : dims) n *= d;
        return n;
    }
};

// Cursor over a byte range with the element-tag rules.
struct Reader {
    const uint8_t* p;
    size_t n, pos = 0;
    bool ok = true;
    Reader(const uint8_t* b, size_t len) : p(b), n(len) {}
    bool at_end() const { return pos + 4 > n; }
    // Reads one tag; returns the payload span; advances past the padded payload.
    bool element(uint32_t& type, const uint8_t*& data, uint32_t& nbytes) {
        if (pos + 8 > n) return ok = false;
        uint32_t w0, w1;
        memcpy(&w0, p + pos, 4);
        memcpy(&w1, p + pos + 4, 4);
        if (w0 >> 16) {  // small element: type and byte count in one word, data in the next 4 bytes
            type = w0 & 0xffff;
            nbytes = w0 >> 16;
            if (nbytes > 4) return ok = false;
            data = p + pos + 4;
            pos += 8;
            return true;
        }
        type = w0;
        nbytes = w1;
        if (pos + 8 + (size_t)nbytes > n) return ok = false;
        data = p + pos + 8;
        size_t adv = 8 + (size_t)nbytes;
        if (type != miCOMPRESSED) adv = (adv + 7) & ~(size_t)7;
        pos = adv + pos > n ? n : pos + adv;
        return true;
    }
};

bool inflate_all(const uint8_t* src, size_t len, std::vector<uint8_t>& out) {
    z_stream zs;
    memset(&zs, 0, sizeof zs);
    if (inflateInit(&zs) != Z_OK) return false;
    out.resize(len * 4 + 1024);
    zs.next_in = const_cast<Bytef*>(src);
    zs.avail_in = (uInt)len;
    int rc = Z_OK;
    while (rc != Z_STREAM_END) {
        if (zs.total_out == out.size()) out.resize(out.size() * 2);
        zs.next_out = out.data() + zs.total_out;
        zs.avail_out = (uInt)(out.size() - zs.total_out);
        rc = inflate(&zs, Z_NO_FLUSH);
        if (rc == Z_BUF_ERROR && zs.avail_in == 0) break;  // truncated stream
        if (rc != Z_OK && rc != Z_STREAM_END && rc != Z_BUF_ERROR) break;
    }
    out.resize(zs.total_out);
    inflateEnd(&zs);
    return rc == Z_STREAM_END;
}

bool parse_matrix(const uint8_t* data, uint32_t nbytes, Var& v, std::string& err) {
    Reader r(data, nbytes);
    uint32_t t, nb;
    const uint8_t* d;
    if (!r.element(t, d, nb) || t != miUINT32 || nb < 8) {
        err = "array flags missing";
        return false;
    }
    uint32_t flags;
    memcpy(&flags, d, 4);
    v.cls = (int)(flags & 0xff);
    v.complex = (flags & 0x800) != 0;
    v.logical = (flags & 0x200) != 0;
    if (v.cls != FKADJ_MX_OPAQUE) {
        if (!r.element(t, d, nb) || t != miINT32 || nb < 8) {
            err = "dimensions missing";
            return false;
        }
        for (uint32_t k = 0; k < nb / 4; ++k) {
            int32_t x;
            memcpy(&x, d + 4 * k, 4);
            if (x < 0) {
                err = "negative dimension";
                return false;
            }
            v.dims.push_back(x);
        }
    }
    if (!r.element(t, d, nb) || (t != miINT8 && t != miUINT8)) {
        err = "array name missing";
        return false;
    }
    v.name.assign((const char*)d, nb);
    auto take = [&](Part& part) {
        if (!r.element(t, d, nb) || (mi_size(t) == 0) || nb % mi_size(t)) return false;
        part.type = t;
        part.bytes.assign(d, d + nb);
        return true;
    };
    if (v.cls == FKADJ_MX_SPARSE) {
        if (!take(v.ir) || !take(v.jc) || !take(v.re) || (v.complex && !take(v.im))) {
            err = "sparse parts missing in '" + v.name + "'";
            return false;
        }
        v.readable = v.dims.size() == 2 && !v.complex && v.jc.count() == v.dims[1] + 1;
    } else if (v.cls == FKADJ_MX_CHAR || (v.cls >= FKADJ_MX_DOUBLE && v.cls <= FKADJ_MX_UINT64)) {
        if (v.numel() > 0 || !r.at_end()) {
            if (!take(v.re) || (v.complex && !take(v.im))) {
                err = "data missing in '" + v.name + "'";
                return false;
            }
        }
        v.readable = !v.complex && v.re.count() == v.numel();
    }
    return true;  // cells, structs, objects, function handles: listed only
}

}  // namespace

struct fkadj_mat {
    std::vector<Var> vars;
    const Var* find(const char* name) const {
        if (!name) return nullptr;
        for (const Var& v : vars)
            if (v.name == name) return &v;
        return nullptr;
    }
};

struct fkadj_matw {
    std::string path;
    bool compress = false;
    std::vector<uint8_t> body;
};

namespace {

const Var* need(const fkadj_mat* m, const char* name, bool sparse) {
    const Var* v = m ? m->find(name) : nullptr;
    if (!v) {
        set_error(std::string("MAT variable '") + (name ? name : "(null)") + "' not found");
        return nullptr;
    }
    if (!v->readable || (sparse != (v->cls == FKADJ_MX_SPARSE))) {
        set_error("MAT variable '" + v->name + "' is not a real " +
                  (sparse ? "sparse matrix" : "dense array"));
        return nullptr;
    }
    return v;
}

}  // namespace

extern "C" {

fkadj_status fkadj_mat_open(const char* path, fkadj_mat** out) {
    if (!path || !out) {
        set_error("fkadj_mat_open: null argument");
        return FKADJ_ERR_ARG;
    }
    *out = nullptr;
    FILE* f = fopen(path, "rb");
    if (!f) {
        set_error(std::string("cannot open ") + path);
        return FKADJ_ERR_ARG;
    }
    std::vector<uint8_t> buf;
    uint8_t chunk[1 << 16];
    size_t got;
    while ((got = fread(chunk, 1, sizeof chunk, f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
    fclose(f);
    if (buf.size() < 128 || memcmp(buf.data(), "MATLAB 5.0 MAT-file", 19) != 0) {
        set_error(std::string(path) + " is not a level-5 MAT file");
        return FKADJ_ERR_ARG;
    }
    if (buf[126] != 'I' || buf[127] != 'M') {
        set_error(std::string(path) + ": only little-endian MAT files are supported");
        return FKADJ_ERR_ARG;
    }
    std::unique_ptr<fkadj_mat> m(new fkadj_mat);
    Reader r(buf.data() + 128, buf.size() - 128);
    std::string err;
    while (!r.at_end()) {
        uint32_t t, nb;
        const uint8_t* d;
        if (!r.element(t, d, nb)) {
            set_error(std::string(path) + ": truncated element");
            return FKADJ_ERR_ARG;
        }
        std::vector<uint8_t> inflated;
        if (t == miCOMPRESSED) {
            if (!inflate_all(d, nb, inflated)) {
                set_error(std::string(path) + ": corrupt compressed element");
                return FKADJ_ERR_ARG;
            }
            Reader ri(inflated.data(), inflated.size());
            if (!ri.element(t, d, nb)) {
                set_error(std::string(path) + ": empty compressed element");
                return FKADJ_ERR_ARG;
            }
        }
        if (t != miMATRIX) continue;  // other top-level elements carry no variable
        Var v;
        if (!parse_matrix(d, nb, v, err)) {
            set_error(std::string(path) + ": " + err);
            return FKADJ_ERR_ARG;
        }
        m->vars.push_back(std::move(v));
    }
    *out = m.release();
    return FKADJ_OK;
}

void fkadj_mat_close(fkadj_mat* m) { delete m; }

int fkadj_mat_count(const fkadj_mat* m) { return m ? (int)m->vars.size() : 0; }

const char* fkadj_mat_name(const fkadj_mat* m, int i) {
    if (!m || i < 0 || i >= (int)m->vars.size()) return nullptr;
    return m->vars[i].name.c_str();
}

fkadj_status fkadj_mat_info(const fkadj_mat* m, const char* name, int* mx_class, int* ndims,
                            int64_t* dims, int maxdims, int64_t* numel, int64_t* nnz,
                            int* flags) {
    const Var* v = m ? m->find(name) : nullptr;
    if (!v) {
        set_error(std::string("MAT variable '") + (name ? name : "(null)") + "' not found");
        return FKADJ_ERR_ARG;
    }
    if (mx_class) *mx_class = v->cls;
    if (ndims) *ndims = (int)v->dims.size();
    if (dims)
        for (int k = 0; k < maxdims && k < (int)v->dims.size(); ++k) dims[k] = v->dims[k];
    if (numel) *numel = v->numel();
    if (nnz) {
        int64_t z = 0;
        if (v->cls == FKADJ_MX_SPARSE && v->readable) v->jc.int_at(v->jc.count() - 1, z);
        *nnz = z;
    }
    if (flags) *flags = (v->complex ? 1 : 0) | (v->logical ? 2 : 0) | (v->readable ? 4 : 0);
    return FKADJ_OK;
}

fkadj_status fkadj_mat_read_double(const fkadj_mat* m, const char* name, double* out, int64_t n) {
    const Var* v = need(m, name, false);
    if (!v) return FKADJ_ERR_ARG;
    if (!out || n != v->numel()) {
        set_error("MAT variable '" + v->name + "' has " + std::to_string(v->numel()) +
                  " elements, " + std::to_string(n) + " requested");
        return FKADJ_ERR_ARG;
    }
    for (int64_t i = 0; i < n; ++i) out[i] = v->re.at(i);
    return FKADJ_OK;
}

fkadj_status fkadj_mat_read_int32(const fkadj_mat* m, const char* name, int32_t* out, int64_t n) {
    const Var* v = need(m, name, false);
    if (!v) return FKADJ_ERR_ARG;
    if (!out || n != v->numel()) {
        set_error("MAT variable '" + v->name + "' has " + std::to_string(v->numel()) +
                  " elements, " + std::to_string(n) + " requested");
        return FKADJ_ERR_ARG;
    }
    for (int64_t i = 0; i < n; ++i) {
        int64_t x;
        if (!v->re.int_at(i, x) || x < INT32_MIN || x > INT32_MAX) {
            set_error("MAT variable '" + v->name + "' element " + std::to_string(i) +
                      " is not an int32 value");
            return FKADJ_ERR_ARG;
        }
        out[i] = (int32_t)x;
    }
    return FKADJ_OK;
}

fkadj_status fkadj_mat_read_string(const fkadj_mat* m, const char* name, char* out, int64_t cap) {
    const Var* v = need(m, name, false);
    if (!v) return FKADJ_ERR_ARG;
    const int64_t n = v->numel();
    if (!out || cap < n + 1) {
        set_error("MAT variable '" + v->name + "' needs " + std::to_string(n + 1) + " bytes");
        return FKADJ_ERR_ARG;
    }
    for (int64_t i = 0; i < n; ++i) {
        const double c = v->re.at(i);
        out[i] = (c >= 1 && c < 128) ? (char)c : '?';
    }
    out[n] = '\0';
    return FKADJ_OK;
}

fkadj_status fkadj_mat_read_sparse(const fkadj_mat* m, const char* name, int64_t* colptr,
                                   int64_t* rowidx, double* val) {
    const Var* v = need(m, name, true);
    if (!v) return FKADJ_ERR_ARG;
    const int64_t ncols = v->dims[1], nrows = v->dims[0];
    if (!colptr) {
        set_error("fkadj_mat_read_sparse: null colptr");
        return FKADJ_ERR_ARG;
    }
    for (int64_t c = 0; c <= ncols; ++c) {
        if (!v->jc.int_at(c, colptr[c]) || colptr[c] < 0 || (c && colptr[c] < colptr[c - 1])) {
            set_error("MAT sparse '" + v->name + "': bad column pointer");
            return FKADJ_ERR_ARG;
        }
    }
    const int64_t nnz = colptr[ncols];
    if (nnz > v->ir.count() || (nnz > v->re.count() && !v->logical)) {
        set_error("MAT sparse '" + v->name + "': fewer stored entries than jc says");
        return FKADJ_ERR_ARG;
    }
    if (nnz && (!rowidx || !val)) {
        set_error("fkadj_mat_read_sparse: null rowidx or val");
        return FKADJ_ERR_ARG;
    }
    for (int64_t k = 0; k < nnz; ++k) {
        if (!v->ir.int_at(k, rowidx[k]) || rowidx[k] < 0 || rowidx[k] >= nrows) {
            set_error("MAT sparse '" + v->name + "': row index out of range");
            return FKADJ_ERR_ARG;
        }
        // a logical sparse matrix may omit its (all-true) values
        val[k] = k < v->re.count() ? v->re.at(k) : 1.0;
    }
    return FKADJ_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- writer
namespace {

void put32(std::vector<uint8_t>& b, uint32_t x) {
    uint8_t t[4];
    memcpy(t, &x, 4);
    b.insert(b.end(), t, t + 4);
}

void pad8(std::vector<uint8_t>& b) {
    while (b.size() % 8) b.push_back(0);
}

// One sub-element: small form when it fits in 4 bytes.
void sub(std::vector<uint8_t>& b, uint32_t type, const void* data, size_t nbytes) {
    if (nbytes <= 4 && nbytes > 0) {
        put32(b, (uint32_t)(nbytes << 16) | type);
        uint8_t t[4] = {0, 0, 0, 0};
        memcpy(t, data, nbytes);
        b.insert(b.end(), t, t + 4);
        return;
    }
    put32(b, type);
    put32(b, (uint32_t)nbytes);
    const uint8_t* d = (const uint8_t*)data;
    if (nbytes) b.insert(b.end(), d, d + nbytes);
    pad8(b);
}

void header(std::vector<uint8_t>& b, uint32_t cls, uint32_t nzmax, int64_t rows, int64_t cols,
            const char* name) {
    const uint32_t flags[2] = {cls, nzmax};
    sub(b, miUINT32, flags, 8);
    const int32_t dims[2] = {(int32_t)rows, (int32_t)cols};
    sub(b, miINT32, dims, 8);
    sub(b, miINT8, name, strlen(name));
}

fkadj_status finish(fkadj_matw* w, std::vector<uint8_t>& m) {
    std::vector<uint8_t> el;
    put32(el, miMATRIX);
    put32(el, (uint32_t)m.size());
    el.insert(el.end(), m.begin(), m.end());
    if (!w->compress) {
        w->body.insert(w->body.end(), el.begin(), el.end());
        return FKADJ_OK;
    }
    uLongf zlen = compressBound((uLong)el.size());
    std::vector<uint8_t> z(zlen);
    if (compress2(z.data(), &zlen, el.data(), (uLong)el.size(), 6) != Z_OK) {
        set_error("zlib compression failed");
        return FKADJ_ERR_NOMEM;
    }
    put32(w->body, miCOMPRESSED);
    put32(w->body, (uint32_t)zlen);
    w->body.insert(w->body.end(), z.begin(), z.begin() + zlen);
    return FKADJ_OK;
}

bool bad_name(const char* name) {
    if (!name || !*name || strlen(name) > 63) return true;
    for (const char* c = name; *c; ++c)
        if (!(isalnum((unsigned char)*c) || *c == '_')) return true;
    return !isalpha((unsigned char)name[0]);
}

bool dims_ok(int64_t rows, int64_t cols) {
    return rows >= 0 && cols >= 0 && rows <= INT32_MAX && cols <= INT32_MAX;
}

}  // namespace

extern "C" {

fkadj_status fkadj_matw_open(const char* path, int compress, fkadj_matw** out) {
    if (!path || !out) {
        set_error("fkadj_matw_open: null argument");
        return FKADJ_ERR_ARG;
    }
    fkadj_matw* w = new fkadj_matw;
    w->path = path;
    w->compress = compress != 0;
    *out = w;
    return FKADJ_OK;
}

fkadj_status fkadj_matw_dense(fkadj_matw* w, const char* name, int mx_class, int64_t rows,
                              int64_t cols, const void* data) {
    if (!w || bad_name(name) || !dims_ok(rows, cols) || (!data && rows * cols != 0)) {
        set_error("fkadj_matw_dense: bad writer, name, dimensions or data");
        return FKADJ_ERR_ARG;
    }
    uint32_t type;
    size_t es;
    switch (mx_class) {
        case FKADJ_MX_DOUBLE: type = miDOUBLE; es = 8; break;
        case FKADJ_MX_INT32: type = miINT32; es = 4; break;
        case FKADJ_MX_INT16: type = miINT16; es = 2; break;
        case FKADJ_MX_UINT8: type = miUINT8; es = 1; break;
        default:
            set_error("fkadj_matw_dense: class must be double, int32, int16 or uint8");
            return FKADJ_ERR_ARG;
    }
    const size_t nbytes = (size_t)(rows * cols) * es;
    if (nbytes > 0xfffff000u) {
        set_error("fkadj_matw_dense: array exceeds the 4 GiB element limit of the format");
        return FKADJ_ERR_ARG;
    }
    std::vector<uint8_t> m;
    header(m, (uint32_t)mx_class, 0, rows, cols, name);
    sub(m, type, data, nbytes);
    return finish(w, m);
}

fkadj_status fkadj_matw_string(fkadj_matw* w, const char* name, const char* s) {
    if (!w || bad_name(name) || !s) {
        set_error("fkadj_matw_string: bad writer, name or string");
        return FKADJ_ERR_ARG;
    }
    const size_t n = strlen(s);
    std::vector<uint16_t> u(n);
    for (size_t i = 0; i < n; ++i) u[i] = (unsigned char)s[i];
    std::vector<uint8_t> m;
    header(m, FKADJ_MX_CHAR, 0, n ? 1 : 0, (int64_t)n, name);
    sub(m, miUINT16, u.data(), 2 * n);
    return finish(w, m);
}

fkadj_status fkadj_matw_sparse(fkadj_matw* w, const char* name, int64_t rows, int64_t cols,
                               const int64_t* colptr, const int64_t* rowidx, const double* val) {
    if (!w || bad_name(name) || !dims_ok(rows, cols) || !colptr || colptr[0] != 0) {
        set_error("fkadj_matw_sparse: bad writer, name, dimensions or column pointer");
        return FKADJ_ERR_ARG;
    }
    const int64_t nnz = colptr[cols];
    if (nnz < 0 || nnz > INT32_MAX || (nnz && (!rowidx || !val))) {
        set_error("fkadj_matw_sparse: bad nnz or null arrays");
        return FKADJ_ERR_ARG;
    }
    std::vector<int32_t> ir((size_t)std::max<int64_t>(nnz, 1), 0), jc((size_t)cols + 1);
    for (int64_t c = 0; c <= cols; ++c) {
        if (c && (colptr[c] < colptr[c - 1])) {
            set_error("fkadj_matw_sparse: column pointer decreases");
            return FKADJ_ERR_ARG;
        }
        jc[c] = (int32_t)colptr[c];
    }
    for (int64_t k = 0; k < nnz; ++k) {
        if (rowidx[k] < 0 || rowidx[k] >= rows) {
            set_error("fkadj_matw_sparse: row index out of range");
            return FKADJ_ERR_ARG;
        }
        ir[k] = (int32_t)rowidx[k];
    }
    const double zero = 0.0;
    std::vector<uint8_t> m;
    const uint32_t nzmax = (uint32_t)std::max<int64_t>(nnz, 1);
    header(m, FKADJ_MX_SPARSE, nzmax, rows, cols, name);
    sub(m, miINT32, ir.data(), 4 * (size_t)nzmax);
    sub(m, miINT32, jc.data(), 4 * ((size_t)cols + 1));
    sub(m, miDOUBLE, nnz ? (const void*)val : (const void*)&zero, 8 * (size_t)nzmax);
    return finish(w, m);
}

fkadj_status fkadj_matw_close(fkadj_matw* w) {
    if (!w) {
        set_error("fkadj_matw_close: null writer");
        return FKADJ_ERR_ARG;
    }
    std::unique_ptr<fkadj_matw> hold(w);
    char text[117];
    memset(text, ' ', sizeof text);
    const time_t now = time(nullptr);
    char when[64];
    strftime(when, sizeof when, "%a %b %d %H:%M:%S %Y", gmtime(&now));
    const int k = snprintf(text, sizeof text,
                           "MATLAB 5.0 MAT-file, Platform: GLNXA64, Created on: %s by libfkadj",
                           when);
    if (k >= 0 && k < (int)sizeof text) text[k] = ' ';
    uint8_t head[128];
    memcpy(head, text, 116);
    memset(head + 116, 0, 8);  // no subsystem data
    head[124] = 0x00;
    head[125] = 0x01;  // version 0x0100, written little-endian
    head[126] = 'I';
    head[127] = 'M';
    FILE* f = fopen(w->path.c_str(), "wb");
    if (!f) {
        set_error("cannot create " + w->path);
        return FKADJ_ERR_ARG;
    }
    bool ok = fwrite(head, 1, 128, f) == 128 &&
              fwrite(w->body.data(), 1, w->body.size(), f) == w->body.size();
    ok = (fclose(f) == 0) && ok;
    if (!ok) {
        set_error("write failed: " + w->path);
        return FKADJ_ERR_ARG;
    }
    return FKADJ_OK;
}

}  // extern "C"
