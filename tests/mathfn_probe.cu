// Test probe (built by tests/test_gpu_mathfn.py): evaluates the kernels' own
// reciprocal next to the IEEE quotient, and the kernels' exponential (the form
// FKADJ_OWN_EXP selects at build time) next to CUDA's exp, on the same inputs.
#include <cuda_runtime.h>

#include "../adjoint-optimization_b200/csrc/fk_device.cuh"

__global__ void k_rcp_probe(const double* __restrict__ x, double* __restrict__ own, double* __restrict__ ieee,
                            long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) {
        own[i] = fkadj::own_rcp(x[i]);
        ieee[i] = 1.0 / x[i];
    }
}

// Host entry: n inputs from host memory, both results back to host memory.
// Returns a cudaError_t value (0 on success).
extern "C" int probe_rcp(const double* hx, double* hown, double* hieee, long long n) {
    if (n <= 0) return 0;
    double* d = nullptr;
    const size_t bytes = (size_t)n * sizeof(double);
    cudaError_t e = cudaMalloc(&d, 3 * bytes);
    if (e) return (int)e;
    if (!(e = cudaMemcpy(d, hx, bytes, cudaMemcpyHostToDevice))) {
        const int nt = 256;
        const long long nb = (n + nt - 1) / nt;
        k_rcp_probe<<<(unsigned)nb, nt>>>(d, d + n, d + 2 * n, n);
        if (!(e = cudaGetLastError()) && !(e = cudaMemcpy(hown, d + n, bytes, cudaMemcpyDeviceToHost)))
            e = cudaMemcpy(hieee, d + 2 * n, bytes, cudaMemcpyDeviceToHost);
    }
    cudaFree(d);
    return (int)e;
}

__global__ void k_exp_probe(const double* __restrict__ x, double* __restrict__ own, double* __restrict__ ref,
                            long long n) {
    fkadj::exp_table_init();
    __syncthreads();
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) {
        own[i] = fkadj::fk_exp(x[i]);
        ref[i] = exp(x[i]);
    }
}

// The same for the exponential.
extern "C" int probe_exp(const double* hx, double* hown, double* href, long long n) {
    if (n <= 0) return 0;
    double* d = nullptr;
    const size_t bytes = (size_t)n * sizeof(double);
    cudaError_t e = cudaMalloc(&d, 3 * bytes);
    if (e) return (int)e;
    if (!(e = cudaMemcpy(d, hx, bytes, cudaMemcpyHostToDevice))) {
        const int nt = 256;
        const long long nb = (n + nt - 1) / nt;
        k_exp_probe<<<(unsigned)nb, nt>>>(d, d + n, d + 2 * n, n);
        if (!(e = cudaGetLastError()) && !(e = cudaMemcpy(hown, d + n, bytes, cudaMemcpyDeviceToHost)))
            e = cudaMemcpy(href, d + 2 * n, bytes, cudaMemcpyDeviceToHost);
    }
    cudaFree(d);
    return (int)e;
}
