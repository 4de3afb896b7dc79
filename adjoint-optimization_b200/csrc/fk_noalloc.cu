// fk_noalloc.cu -- the z.gh reduction of the gradient for callers that cannot
// allocate device memory.
//
// Who needs it: code whose device memory belongs to another allocator (a
// framework's caching allocator or a memory pool that reserved the GPU up
// front, where an extra cudaMalloc fails or forces a device-wide
// synchronisation), and latency-critical loops that must not call
// cudaMalloc/cudaFree between launches.  They hold the adjoint state and gh
// themselves and only need the inner product z_u . gh that the reference
// takes once per backward step (zgh_dot_partial + vec_sum,
// src/cuda/fk_grad_Et_mono_PARAMETERS.cu:1457-1483 and 1553-1561).
//
// How: the per-sub-block partial sums live in a file-scope device array of a
// fixed size instead of a buffer from cudaMalloc.  Host code cannot use the
// array's name as a device address (it denotes a host-side stand-in), so the
// first call on each device, with that device current, resolves the address
// with cudaGetSymbolAddress and caches it; that first call should therefore
// come before any stream capture.  The cached address belongs to the device's
// primary context of that moment: after cudaDeviceReset (or any teardown and
// re-creation of the primary context) it is stale, and the entry point must
// not be called again in the process.  Every later call on the device re-uses the
// same array: calls that overlap on the GPU (other streams, other host
// threads) race on it and must be serialised by the caller.  Each call writes
// every partial it later reads, so nothing has to start at zero and the array
// keeps the last call's values.
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "../../include/fkadj.h"

namespace fkadj {
void set_error(const std::string& msg);
}

namespace {

// 16x16 sub-blocks the scratch holds: grids up to 65536 sub-blocks
// (16.7 M cells, e.g. 4096 x 4096); 512 KiB per device.
constexpr int kNoAllocMaxSubblocks = FKADJ_NOALLOC_MAX_SUBBLOCKS;

static __device__ __align__(256) double g_zgh_scratch[kNoAllocMaxSubblocks];

std::mutex g_mu;
double* g_scratch_ptr[64];
bool g_scratch_ready[64];

// One warp per 16x16 sub-block of the dense row-major grid; lane l adds the
// 8 cells of half-row l in column order, then a shuffle tree.  NaN products
// (holes) and cells past the grid edge count as 0.
__global__ void __launch_bounds__(32) k_zgh_partials_dense(const double* __restrict__ zu,
                                                           const double* __restrict__ gh, int nrows, int ncols,
                                                           int nsbx, double* __restrict__ part) {
    const int b = blockIdx.x, by = b / nsbx, bx = b - by * nsbx;
    const int lane = threadIdx.x;
    const int r = by * 16 + (lane >> 1), c0 = bx * 16 + (lane & 1) * 8;
    double s = 0.0;
    if (r < nrows) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int c = c0 + k;
            if (c < ncols) {
                const long long o = (long long)r * ncols + c;
                const double t = zu[o] * gh[o];
                if (!isnan(t)) s += t;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) part[b] = s;
}

// out = sum of part[0..n) in a fixed order (one block of 256 threads).
__global__ void __launch_bounds__(256) k_zgh_total(const double* __restrict__ part, int n,
                                                   double* __restrict__ out) {
    __shared__ double red[8];
    double v = 0.0;
    for (int k = threadIdx.x; k < n; k += 256) v += part[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < 8; ++w) s += red[w];
        *out = s;
    }
}

// Device address of the scratch array on the current device (resolved once).
fkadj_status scratch_for_current_device(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        fkadj::set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        return FKADJ_ERR_CUDA;
    }
    if (dev < 0 || dev >= 64) {
        fkadj::set_error("device ordinal out of range for the no-allocation scratch");
        return FKADJ_ERR_NODEVICE;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ready[dev]) {
        double* p = nullptr;
        e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_zgh_scratch);
        if (e != cudaSuccess) {
            fkadj::set_error(std::string("cudaGetSymbolAddress(no-allocation scratch): ") + cudaGetErrorString(e));
            return FKADJ_ERR_CUDA;
        }
        g_scratch_ptr[dev] = p;
        g_scratch_ready[dev] = true;
    }
    *out = g_scratch_ptr[dev];
    return FKADJ_OK;
}

}  // namespace

extern "C" fkadj_status fkadj_zgh_dot_noalloc(const double* d_zu, const double* d_gh, int nrows, int ncols,
                                              double* d_out, void* stream) {
    if (!d_zu || !d_gh || !d_out || nrows < 1 || ncols < 1) {
        fkadj::set_error("fkadj_zgh_dot_noalloc: null pointer or empty grid");
        return FKADJ_ERR_ARG;
    }
    const int nsbx = (ncols + 15) / 16, nsby = (nrows + 15) / 16;
    if ((long long)nsbx * nsby > kNoAllocMaxSubblocks) {
        fkadj::set_error("fkadj_zgh_dot_noalloc: grid needs " + std::to_string((long long)nsbx * nsby) +
                         " 16x16 sub-blocks, more than the fixed scratch holds (" +
                         std::to_string(kNoAllocMaxSubblocks) + ", i.e. 16.7 M cells)");
        return FKADJ_ERR_ARG;
    }
    double* scratch = nullptr;
    fkadj_status s = scratch_for_current_device(&scratch);
    if (s != FKADJ_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nsb = nsbx * nsby;
    k_zgh_partials_dense<<<nsb, 32, 0, st>>>(d_zu, d_gh, nrows, ncols, nsbx, scratch);
    k_zgh_total<<<1, 256, 0, st>>>(scratch, nsb, d_out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fkadj::set_error(std::string("fkadj_zgh_dot_noalloc launch: ") + cudaGetErrorString(e));
        return FKADJ_ERR_CUDA;
    }
    return FKADJ_OK;
}
