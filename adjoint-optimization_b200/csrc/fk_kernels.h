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

int tile_count();
TileShape tile_shape(int tile);
int tiles_of(int tile, const DevGrid& g);
cudaError_t kernels_init();

cudaError_t launch_fwd_step(int tile, const DevModel& P, const DevGrid& g, const double* yin, double* yout,
                            const double* gh, double E0, double Eh, double E1, cudaStream_t st,
                            double* stages = nullptr);
// The z.gh style reductions write one partial per 16x16 sub-block of the
// grid's lattice (nsbx x nsby, covering the 64-padded grid); sub-blocks no
// tile covers are never written and must be zero.
void subblock_lattice(const DevGrid& g, int* nsbx, int* nsby);
cudaError_t launch_adj_exact(int tile, const DevModel& P, const DevGrid& g, const double* lam, double* lamout,
                             const double* y, const double* stages, const uint8_t* wc, const double* gh,
                             double* r1, double* r23, double* r4, int nsbx, cudaStream_t st);
cudaError_t launch_adj_mid(int tile, const DevModel& P, const DevGrid& g, const double* ya, const double* yb,
                           const double* gh, double* yh, double Ea, double Eb, double E3, const HermiteW& hw,
                           cudaStream_t st, const double* fin = nullptr, double* fout = nullptr,
                           double* jh = nullptr);
// jb: cached J(y_i) (null = evaluate), jh: cached J(yh) (null = evaluate),
// ja: where J(y_{i-1}) is stored for the next step (null = not kept).
cudaError_t launch_adj_step(int tile, const DevModel& P, const DevGrid& g, const double* z, double* zout,
                            const double* yb, const double* yh, const double* ya, const uint8_t* wc,
                            const double* gh, double* row, int nsbx, cudaStream_t st, const double* jb = nullptr,
                            const double* jh = nullptr, double* ja = nullptr);
cudaError_t launch_dot_gh(const DevGrid& g, const double* z, const double* gh, double* row, int nsbx, int nsby,
                          cudaStream_t st);
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
