// FP64 inner products of FP32 arrays on the GPU: the reduction behind every
// dot-product test of the operator pairs (F/include/operator.h:50-88 takes
// <F m, d> and <m, F* d> with SEP vector dot products).
//
// Each product a[i]*b[i] is formed exactly in FP64 (a float times a float is
// exact in double), accumulated per thread in FP64 over a grid-stride range,
// then summed by a fixed-shape tree: per warp by shuffles, per block through
// shared memory, and the per-block partials by one block in index order. The
// grid shape depends only on n, so the result is bitwise reproducible from run
// to run for the same inputs on the same GPU model.
#include <algorithm>
#include <cstdio>

#include <cuda_runtime.h>

#include "aio_b200.h"

#define AIO_API extern "C" __attribute__((visibility("default")))

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 148 * 8;  // 8 resident blocks on each of the 148 SMs

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double warp_part[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) warp_part[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (warp == 0) {
        s = lane < kThreads / 32 ? warp_part[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    return s;  // valid in thread 0
}

__global__ void __launch_bounds__(kThreads) k_dot_partial(const float* __restrict__ a, const float* __restrict__ b,
                                                          long long n, double* __restrict__ part) {
    double acc = 0.0;
    const long long stride = (long long)gridDim.x * kThreads;
    for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride)
        acc += (double)__ldg(a + i) * (double)__ldg(b + i);
    const double s = block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kThreads) k_dot_final(const double* __restrict__ part, int nPart,
                                                        double* __restrict__ out) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < nPart; i += kThreads) acc += part[i];
    const double s = block_sum(acc);
    if (threadIdx.x == 0) *out = s;
}

int fail(int code, const char* what, cudaError_t e) {
    std::fprintf(stderr, "aio_dot_f64: %s: %s\n", what, cudaGetErrorString(e));
    return code;
}

}  // namespace

AIO_API int aio_dot_f64(int device, int memSpace, long long n, const float* a, const float* b, double* result) {
    if (!result || n < 0 || (n > 0 && (!a || !b)) || (memSpace != AIO_MEM_HOST && memSpace != AIO_MEM_DEVICE))
        return AIO_ERR_ARGUMENT;
    *result = 0.0;
    if (n == 0) return AIO_OK;
    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return fail(AIO_ERR_CUDA, "cudaGetDevice", e);
    if ((e = cudaSetDevice(device)) != cudaSuccess) return fail(AIO_ERR_CUDA, "cudaSetDevice", e);
    const int blocks = (int)std::min<long long>(kMaxBlocks, (n + kThreads - 1) / kThreads);
    float* da = nullptr;
    float* db = nullptr;
    double* dpart = nullptr;
    int rc = AIO_OK;
    const float* pa = a;
    const float* pb = b;
    cudaStream_t st = nullptr;
    do {
        if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) {
            rc = fail(AIO_ERR_CUDA, "cudaStreamCreate", e);
            break;
        }
        if ((e = cudaMalloc(&dpart, sizeof(double) * (blocks + 1))) != cudaSuccess) {
            rc = fail(AIO_ERR_MEMORY, "cudaMalloc", e);
            break;
        }
        if (memSpace == AIO_MEM_HOST) {
            if ((e = cudaMalloc(&da, sizeof(float) * n)) != cudaSuccess ||
                (e = cudaMalloc(&db, sizeof(float) * n)) != cudaSuccess) {
                rc = fail(AIO_ERR_MEMORY, "cudaMalloc", e);
                break;
            }
            if ((e = cudaMemcpyAsync(da, a, sizeof(float) * n, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
                (e = cudaMemcpyAsync(db, b, sizeof(float) * n, cudaMemcpyHostToDevice, st)) != cudaSuccess) {
                rc = fail(AIO_ERR_CUDA, "cudaMemcpyAsync", e);
                break;
            }
            pa = da;
            pb = db;
        }
        k_dot_partial<<<blocks, kThreads, 0, st>>>(pa, pb, n, dpart);
        k_dot_final<<<1, kThreads, 0, st>>>(dpart, blocks, dpart + blocks);
        if ((e = cudaGetLastError()) != cudaSuccess) {
            rc = fail(AIO_ERR_CUDA, "kernel launch", e);
            break;
        }
        if ((e = cudaMemcpyAsync(result, dpart + blocks, sizeof(double), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess) {
            rc = fail(AIO_ERR_CUDA, "result copy", e);
            break;
        }
    } while (false);
    if (st) cudaStreamSynchronize(st);
    cudaFree(da);
    cudaFree(db);
    cudaFree(dpart);
    if (st) cudaStreamDestroy(st);
    cudaSetDevice(prev);
    return rc;
}
