// fk_kernels.h -- launchers of the sm_100a kernels (host-callable, C++).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "fk_device.cuh"

namespace fkadj {

struct TileShape {
    int tx, ty, nt;
};

// Hermite weights of the midpoint reconstruction (cu-G:1217-1241, 1295-1298).
struct HermiteW {
    double c3[4];  // cubic at t = 1/3: x0, m0, x1, m1
    double c4[4];  // partial quartic at t = 1/2
    double c2;     // weight of dt*f(y3) in the quartic
};

// ------------------------------------------------------------ batched ticks
// Per-instance constants of a batch (device array).
struct BatchInstance {
    DevModel P;
    DevGrid g;
    const double* gh;
    const uint8_t* wc;
    unsigned* fault;  // the problem's fault word (set when a tile copy's bounded wait expires)
    int nsbx;
};

enum BatchKind { BATCH_FWD = 0, BATCH_MID = 1, BATCH_ADJ_REF = 2, BATCH_ADJ_EXACT = 3, BATCH_ADJ_FUSED = 4 };

// One instance's work of one kind in one tick; it owns tiles
// [tile0, tile0 + ntx*nty) of the tick's launch.  Field use by kind:
//   FWD        a = y_in, out = y_out, stages (or null), E0/E1/E2 = Et[i], Eh[i], Et[i+1]
//   MID        a = y_{i-1}, b = y_i, out = yh, E0/E1/E2 = Et[i-1], Et[i], E(t_{i-1}+dt/3),
//              fin/fout (f carry), jh (J(yh) out)
//   ADJ_REF    a = z, out = z_out, b = y_i, c = yh, d = y_{i-1}, row, jb/jh/ja (J caches)
//   ADJ_EXACT  a = lambda, out = lambda_out, b = y_s, stages, row/row2/row3
//   ADJ_FUSED  a = z, out = z_out, b = y_i, d = y_{i-1}, fa, fin (f(y_i)), fout, row, jb/ja,
//              E0/E1/E2 = Et[i-1], Et[i], E(t_{i-1}+dt/3)
// The three E samples of one step: (E0, Eh, E1) = (Et[i], E(t_i + dt/2),
// Et[i+1]) for the forward step, (Ea, Eb, E3) = (Et[i-1], Et[i], E(t_{i-1} +
// dt/3)) for the adjoint midpoint.  Either by value, or read by the kernel from
// device tables (p[k] non-null), so a captured launch sequence (CUDA graph)
// replays with new samples written into the tables.
struct EStep {
    double v[3];
    const double* p[3];
    __host__ __device__ static EStep values(double a, double b, double c) { return {{a, b, c}, {nullptr, nullptr, nullptr}}; }
    __host__ __device__ static EStep table(const double* a, const double* b, const double* c) {
        return {{0.0, 0.0, 0.0}, {a, b, c}};
    }
    __device__ double a() const { return p[0] ? *p[0] : v[0]; }
    __device__ double b() const { return p[1] ? *p[1] : v[1]; }
    __device__ double c() const { return p[2] ? *p[2] : v[2]; }
};

struct BatchItem {
    int inst, tile0, ntx, kind;
    const double *a, *b, *c, *d;
    double *out, *stages;
    double E0, E1, E2;
    const double* fin;
    double *fout, *jh;
    const double* fa;  // midpoint: kept f(ya) (null = evaluate)
    double* k1;        // forward: where k1 = f(y) is kept (null = not kept)
    const double* jb;
    double* ja;
    double *row, *row2, *row3;
};

constexpr int kBatchMaxItems = 128;

// A tick's work queue for one kernel kind, as the host builds it.
struct BatchTick {
    int n;      // items
    int tiles;  // total tiles
    BatchItem item[kBatchMaxItems];
};

// A tick's work queue of one kernel kind as the kernels read it: n items in
// device memory, `tiles` tiles in all.  With hdr non-null the three numbers
// are read from device memory instead (hdr[0] = n, hdr[1] = tiles, the items
// at items + hdr[2]): a launch captured in a CUDA graph then serves any queue
// written there before it runs.
struct BatchQueue {
    const BatchItem* items;
    int n;
    int tiles;
    const int* hdr = nullptr;
};

cudaError_t launch_batch_fwd(int tile, const BatchInstance* d_inst, const BatchQueue& q, cudaStream_t st);
cudaError_t launch_batch_mid(int tile, const BatchInstance* d_inst, const BatchQueue& q, const HermiteW& hw,
                             cudaStream_t st);
cudaError_t launch_batch_adj(int tile, const BatchInstance* d_inst, const BatchQueue& q, cudaStream_t st);
// fused reference-adjoint steps of a tick; tile: a fused preset (fused_shape)
cudaError_t launch_batch_fused(int tile, const BatchInstance* d_inst, const BatchQueue& q, const HermiteW& hw,
                               cudaStream_t st);

int tile_count();
// The preset the batched kernels run for an autotuned single-instance preset.
int batch_preset(int tile);
TileShape tile_shape(int tile);
int tiles_of(int tile, const DevGrid& g);
cudaError_t kernels_init();
// Reads and clears a problem's fault word d_fault, which the step kernels set
// when one of their bounded waits expires (after synchronising st); *fault != 0
// means the results since the last check are invalid.  Every problem has its
// own word, so problems running at once on other streams or host threads
// neither see nor clear each other's faults.
cudaError_t take_device_fault(cudaStream_t st, unsigned* d_fault, unsigned* fault);

// ty: rows per tile, 0 < ty < the preset's height, or 0 for the preset's
// height (forward step and adjoint midpoint only).  k1 (forward step): where
// k1 = f(y, E0) is kept (a state, null = not kept).  fa (midpoint): f(ya, Ea)
// as kept by the forward step from ya (null = evaluate).  fault: the launching
// problem's fault word (device memory; null = not reported).
cudaError_t launch_fwd_step(int tile, const DevModel& P, const DevGrid& g, const double* yin, double* yout,
                            const double* gh, const EStep& E, cudaStream_t st, unsigned* fault,
                            double* stages = nullptr, int ty = 0, double* k1 = nullptr);
// Programmatic dependent launch for the step kernels issued by this thread
// (on by default; the engine turns it off while it captures a graph).
void set_launch_pdl(bool on);
// Rows per tile that fit grid g into one wave of CTAs of preset `tile` for
// kernel kind 0 (forward step), 1 (adjoint midpoint) or 2 (adjoint step); the
// preset's height when it does not fit.
int balanced_rows(int tile, int kind, const DevGrid& g);
// The z.gh style reductions write one partial per 16x16 sub-block of the
// grid's lattice (nsbx x nsby, covering the 64-padded grid); sub-blocks no
// tile covers are never written and must be zero.  The reference-mode adjoint
// step and launch_dot_gh can instead write one partial per 16-cell row segment
// (segments = true: nsbx x nrows partials per row of results), which lets the
// step's tiles take any number of rows.
void subblock_lattice(const DevGrid& g, int* nsbx, int* nsby);
cudaError_t launch_adj_exact(int tile, const DevModel& P, const DevGrid& g, const double* lam, double* lamout,
                             const double* y, const double* stages, const uint8_t* wc, const double* gh,
                             double* r1, double* r23, double* r4, int nsbx, cudaStream_t st, unsigned* fault);
cudaError_t launch_adj_mid(int tile, const DevModel& P, const DevGrid& g, const double* ya, const double* yb,
                           const double* gh, double* yh, const EStep& E, const HermiteW& hw, cudaStream_t st,
                           unsigned* fault, const double* fin = nullptr, double* fout = nullptr,
                           double* jh = nullptr, int ty = 0, const double* fa = nullptr);
// jb: cached J(y_i) (null = evaluate), jh: cached J(yh) (null = evaluate),
// ja: where J(y_{i-1}) is stored for the next step (null = not kept).
// segments: z.gh partials on the row-segment lattice, with ty rows per tile
// (0 = the preset's height); otherwise on the 16x16 lattice with the preset's
// height.
cudaError_t launch_adj_step(int tile, const DevModel& P, const DevGrid& g, const double* z, double* zout,
                            const double* yb, const double* yh, const double* ya, const uint8_t* wc,
                            const double* gh, double* row, int nsbx, cudaStream_t st, unsigned* fault,
                            const double* jb = nullptr, const double* jh = nullptr, double* ja = nullptr,
                            int ty = 0, bool segments = false);
// Fused reference-adjoint step (k_adj_mid and k_adj_step in one launch):
// z -> zout over step [t_{i-1}, t_i] with ya = y_{i-1}, yb = y_i; fa, fb =
// f(ya, Et[i-1]), f(yb, Et[i]) where kept or carried (null = evaluated), fout
// (null = not kept) receives f(ya) when it was evaluated; E = (Et[i-1], Et[i],
// E(t_{i-1} + dt/3)); jb = cached J_F(y_i)^T (null = evaluated), ja = where
// J_F(y_{i-1})^T is stored for the next step (null = not stored).
// tile: 0 .. fused_count()-1 (fused_shape).
int fused_count();
TileShape fused_shape(int tile);
cudaError_t launch_adj_fused(int tile, const DevModel& P, const DevGrid& g, const double* z, double* zout,
                             const double* ya, const double* yb, const double* fa, const double* fb, double* fout,
                             const uint8_t* wc, const double* gh, const EStep& E, const HermiteW& hw, double* row,
                             int nsbx, const double* jb, double* ja, cudaStream_t st, unsigned* fault);
cudaError_t launch_dot_gh(const DevGrid& g, const double* z, const double* gh, double* row, int nsbx, int nsby,
                          cudaStream_t st, bool segments = false);
cudaError_t launch_sum_rows(const double* partial, int rows, int ntiles, double* out, cudaStream_t st);
cudaError_t launch_scatter(const DevGrid& g, const double* yc, int n_num, const long long* pos, double scale,
                           double* y, cudaStream_t st);
cudaError_t launch_gather(const DevGrid& g, const double* y, int n_num, const long long* pos, double* yc,
                          cudaStream_t st);
int objective_blocks(int n_num);
cudaError_t launch_objective(const double* yc, int n_num, const long long* rowptr, const int* colidx,
                             const double* val, const double gamma[3], double* zc, double* partial,
                             cudaStream_t st);

}  // namespace fkadj
