// FP64 reductions on the GPU: the dot products of the adjoint tests, the data
// misfit and the gradient norms of the FWI loop.  FP32 fields (and the FP64
// vectors of the L-BFGS recursion) are summed in FP64.  The summation order is fixed
// (a grid-stride partial per thread, a shuffle tree per warp, the warps of a
// block in order, the blocks in order), so a result does not change from run to
// run.  The reference forms these sums on the host (pySolver vectors,
// operator.h:50-89 for the dot-product test).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "eio_internal.h"

namespace eio {

namespace {

constexpr int RT = 256;   // threads per block

template <int OP, class T>
__global__ void __launch_bounds__(RT) k_reduce64(const T* __restrict__ x, const T* __restrict__ y,
                                                  long long n, double* __restrict__ partial)
{
    double acc = 0.0;
    const long long stride = (long long)gridDim.x * RT;
    for (long long i = (long long)blockIdx.x * RT + threadIdx.x; i < n; i += stride) {
        const double a = x[i], b = y[i];
        acc += OP == 0 ? a * b : (a - b) * (a - b);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    __shared__ double ws[RT / 32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < RT / 32; w++) s += ws[w];
        partial[blockIdx.x] = s;
    }
}

__global__ void k_sum_blocks(const double* __restrict__ partial, int m, double* __restrict__ out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < m; i++) s += partial[i];
        *out = s;
    }
}

#define RCUDA(x)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (x);                                                                          \
        if (e_ != cudaSuccess) throw Error(EIO_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct DevMem {
    void* p = nullptr;
    ~DevMem() { if (p) cudaFree(p); }
};

// sum over one device-resident range into *out (device), blocks partials in part
template <class T>
void reduce_dev(int op, const T* x, const T* y, long long n, double* part, int nblk, double* out, cudaStream_t st)
{
    if (op == 0) k_reduce64<0, T><<<nblk, RT, 0, st>>>(x, y, n, part);
    else k_reduce64<1, T><<<nblk, RT, 0, st>>>(x, y, n, part);
    k_sum_blocks<<<1, 32, 0, st>>>(part, nblk, out);
    RCUDA(cudaGetLastError());
}

}  // namespace

template <class T>
double reduce64_t(int device, int op, const T* x, const T* y, long long n, bool on_device)
{
    if (op != 0 && op != 1) throw Error(EIO_ERR_ARG, "reduction op must be 0 (dot) or 1 (squared difference)");
    if (n < 0 || (n > 0 && (!x || !y))) throw Error(EIO_ERR_ARG, "reduction: null array or negative length");
    if (n == 0) return 0.0;
    RCUDA(cudaSetDevice(device));
    int nsm = 148;
    RCUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    const int nblk = 4 * nsm;
    cudaStream_t st = nullptr;
    RCUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{st};
    DevMem part, out;
    RCUDA(cudaMalloc(&part.p, sizeof(double) * nblk));
    RCUDA(cudaMalloc(&out.p, sizeof(double)));
    double total = 0.0;
    if (on_device) {
        reduce_dev(op, x, y, n, static_cast<double*>(part.p), nblk, static_cast<double*>(out.p), st);
        RCUDA(cudaMemcpyAsync(&total, out.p, sizeof(double), cudaMemcpyDeviceToHost, st));
        RCUDA(cudaStreamSynchronize(st));
        return total;
    }
    // host arrays: staged through the device in chunks, chunk sums added in order
    const long long chunk = std::min<long long>(n, 1LL << 24);
    DevMem dx, dy;
    RCUDA(cudaMalloc(&dx.p, sizeof(T) * chunk));
    if (y != x) RCUDA(cudaMalloc(&dy.p, sizeof(T) * chunk));
    T* fx = static_cast<T*>(dx.p);
    T* fy = y != x ? static_cast<T*>(dy.p) : fx;
    for (long long i0 = 0; i0 < n; i0 += chunk) {
        const long long m = std::min(chunk, n - i0);
        RCUDA(cudaMemcpyAsync(fx, x + i0, sizeof(T) * m, cudaMemcpyHostToDevice, st));
        if (y != x) RCUDA(cudaMemcpyAsync(fy, y + i0, sizeof(T) * m, cudaMemcpyHostToDevice, st));
        reduce_dev(op, fx, fy, m, static_cast<double*>(part.p), nblk, static_cast<double*>(out.p), st);
        double s = 0.0;
        RCUDA(cudaMemcpyAsync(&s, out.p, sizeof(double), cudaMemcpyDeviceToHost, st));
        RCUDA(cudaStreamSynchronize(st));
        total += s;
    }
    return total;
}

double reduce64(int device, int op, int dtype, const void* x, const void* y, long long n, bool on_device)
{
    if (dtype == 0)
        return reduce64_t(device, op, static_cast<const float*>(x), static_cast<const float*>(y), n, on_device);
    if (dtype == 1)
        return reduce64_t(device, op, static_cast<const double*>(x), static_cast<const double*>(y), n, on_device);
    throw Error(EIO_ERR_ARG, "reduction dtype must be 0 (FP32) or 1 (FP64)");
}

}  // namespace eio
