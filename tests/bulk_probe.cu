// Test probe (built by tests/test_gpu_bulk.py): drives the bulk-copy helpers
// the step kernels load their tile windows with (fk_bulk.cuh) on one CTA.
#include <cuda_runtime.h>

#include "../adjoint-optimization_b200/csrc/fk_bulk.cuh"

using namespace fkadj;

constexpr int RCAP = 40, WIDTH = 72, NT = 256;

// Copies a rows x WIDTH window of three planes into shared memory, posting
// `extra` bytes more than the copies deliver (extra > 0 makes the wait expire),
// then writes the window back densely (3 x rows x WIDTH) and the wait's outcome.
// With cta_mode the wait is the step kernels' bulk_wait_cta: on expiry the CTA
// sets *fault and returns before writing anything.
__global__ void __launch_bounds__(NT) k_bulk_probe(const double* __restrict__ src, int ld, long long plane,
                                                   int rows, unsigned extra, unsigned long long limit_ns,
                                                   double* __restrict__ out, int* __restrict__ status,
                                                   int cta_mode, unsigned* __restrict__ fault) {
    extern __shared__ double4 smem_raw[];
    double* S = reinterpret_cast<double*>(smem_raw);
    __shared__ uint64_t bar;
    const uint32_t b = bulk_begin(&bar);
    __syncthreads();
    bulk_arrive(b, bulk_bytes<WIDTH>(rows) + extra);
    __syncthreads();
    bulk_issue<RCAP, WIDTH, NT>(b, S, src, ld, plane, rows);
    if (cta_mode && !bulk_wait_cta(b, fault, limit_ns)) return;
    const bool ok = cta_mode ? true : bulk_wait(b, limit_ns);
    __syncthreads();
    if (threadIdx.x == 0) *status = ok ? 1 : 0;
    const int per = rows * WIDTH;
    for (int q = threadIdx.x; q < 3 * per; q += NT) {
        const int f = q / per, rem = q - f * per;
        out[q] = S[f * RCAP * WIDTH + rem];
    }
}

// Host entry.  h_src holds 3 planes of rows_alloc x ld doubles; the window
// starts at column col0 (even) of row 0.  Returns a cudaError_t value; *ms is
// the kernel's device time; *h_fault the fault word after the call (cta_mode).
extern "C" int probe_bulk(const double* h_src, int rows_alloc, int ld, int rows, int col0, unsigned extra,
                          unsigned long long limit_ns, double* h_out, int* h_status, float* ms, int cta_mode,
                          unsigned* h_fault) {
    if (rows < 1 || rows > RCAP || rows > rows_alloc || col0 < 0 || col0 + WIDTH > ld || (col0 & 1) || (ld & 1))
        return (int)cudaErrorInvalidValue;
    const long long plane = (long long)rows_alloc * ld;
    const size_t in_bytes = 3 * (size_t)plane * sizeof(double), out_bytes = 3 * (size_t)rows * WIDTH * sizeof(double);
    double *d_src = nullptr, *d_out = nullptr;
    int* d_status = nullptr;
    unsigned* d_fault = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMalloc(&d_src, in_bytes);
    if (!e) e = cudaMalloc(&d_out, out_bytes);
    if (!e) e = cudaMalloc(&d_status, sizeof(int));
    if (!e) e = cudaMalloc(&d_fault, sizeof(unsigned));
    if (!e) e = cudaMemcpy(d_src, h_src, in_bytes, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(d_out, h_out, out_bytes, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemset(d_status, 0xff, sizeof(int));
    if (!e) e = cudaMemset(d_fault, 0, sizeof(unsigned));
    const int smem = 3 * RCAP * WIDTH * (int)sizeof(double);
    if (!e) e = cudaFuncSetAttribute(k_bulk_probe, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (!e) e = cudaEventCreate(&e0);
    if (!e) e = cudaEventCreate(&e1);
    if (!e) e = cudaEventRecord(e0);
    if (!e) {
        k_bulk_probe<<<1, NT, smem>>>(d_src + col0, ld, plane, rows, extra, limit_ns, d_out, d_status, cta_mode,
                                      d_fault);
        e = cudaGetLastError();
    }
    if (!e) e = cudaEventRecord(e1);
    if (!e) e = cudaEventSynchronize(e1);
    if (!e) e = cudaEventElapsedTime(ms, e0, e1);
    if (!e) e = cudaMemcpy(h_out, d_out, out_bytes, cudaMemcpyDeviceToHost);
    if (!e) e = cudaMemcpy(h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (!e) e = cudaMemcpy(h_fault, d_fault, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d_src);
    cudaFree(d_out);
    cudaFree(d_status);
    cudaFree(d_fault);
    return (int)e;
}
