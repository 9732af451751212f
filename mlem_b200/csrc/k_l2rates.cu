// k_l2rates.cu -- what the L2 serves to random addresses: the rates that
// bound the one-pass walk (mlem_measure_l2_rates).
//
// Four kernels over a 64 MB device array (resident in the 126 MB L2), every
// address drawn by a hash so that no two accesses of a warp share a sector:
// float gathers of 4 bytes (one lane each) and of 64-byte rows (4 lanes x 16
// bytes, as the one-pass walk gathers 16 frames), float reductions
// (red.global.add) of 4 bytes and of 64-byte rows (red.v4 by 4 lanes).  Each
// is timed with CUDA events after a warm-up launch.  The one-pass walk gathers
// image values and reduces update values at such addresses; the reduction
// rates bound it.
#include <algorithm>

#include "common.cuh"
#include "mlem_b200.h"

namespace {

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

constexpr uint32_t kRows = 1u << 20;  // 64-byte rows: 64 MB
constexpr int kThreads = 256;
constexpr uint32_t kIters = 512;

__global__ void k_gather4(const float* __restrict__ x, float* __restrict__ sink) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t h = mix32(tid * 0x9e3779b9u + 11u);
    float acc = 0.0f;
    for (uint32_t i = 0; i < kIters; i += 8) {
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            h = mix32(h + j);
            v[j] = __ldg(x + (h & (kRows * 16 - 1)));
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) acc += v[j];
    }
    if (acc == -1.0f) sink[tid] = acc;  // never true (the array is zero): keeps the loads
}

__global__ void k_gather64(const float4* __restrict__ x, float* __restrict__ sink) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t sub = tid & 3;
    uint32_t h = mix32((tid >> 2) * 0x9e3779b9u + 1u);
    float acc = 0.0f;
    for (uint32_t i = 0; i < kIters; i += 4) {
        float4 v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            h = mix32(h + j);
            v[j] = __ldg(x + (size_t)(h & (kRows - 1)) * 4 + sub);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) acc += v[j].x + v[j].y + v[j].z + v[j].w;
    }
    if (acc == -1.0f) sink[tid] = acc;
}

__global__ void k_red4(float* __restrict__ u) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t h = mix32(tid * 0x9e3779b9u + 13u);
    for (uint32_t i = 0; i < kIters / 4; ++i) {
        h = mix32(h + i);
        atomicAdd(u + (h & (kRows * 16 - 1)), 1e-9f);
    }
}

__global__ void k_red64(float4* __restrict__ u) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t sub = tid & 3;
    uint32_t h = mix32((tid >> 2) * 0x9e3779b9u + 7u);
    for (uint32_t i = 0; i < kIters / 4; ++i) {
        h = mix32(h + i);
        atomicAdd(u + (size_t)(h & (kRows - 1)) * 4 + sub, make_float4(1e-9f, 1e-9f, 1e-9f, 1e-9f));
    }
}

}  // namespace

extern "C" int mlem_measure_l2_rates(int device, double* rates) {
    if (!rates) return MLEM_ERR_INVALID;
    int n_sm = 0;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        return MLEM_ERR_CUDA;
    }
    float* a = nullptr;
    float* sink = nullptr;
    const int blocks = std::max(1, n_sm) * 8;
    const size_t threads = (size_t)blocks * kThreads;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStream_t st = nullptr;
    cudaError_t e = cudaMalloc(&a, (size_t)kRows * 64);
    if (e == cudaSuccess) e = cudaMalloc(&sink, threads * 4);
    if (e == cudaSuccess) e = cudaMemset(a, 0, (size_t)kRows * 64);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    // per launch: accesses (gathers or reductions) of the measured width
    const double n_word = (double)threads * kIters, n_row = (double)threads / 4 * kIters;
    const double counts[4] = {n_word, n_row, n_word / 4, n_row / 4};
    for (int k = 0; k < 4 && e == cudaSuccess; ++k) {
        float ms = 0.0f;
        for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {  // a warm-up launch, then the timed one
            if (rep == 1) e = cudaEventRecord(e0, st);
            switch (k) {
                case 0: k_gather4<<<blocks, kThreads, 0, st>>>(a, sink); break;
                case 1: k_gather64<<<blocks, kThreads, 0, st>>>(reinterpret_cast<const float4*>(a), sink); break;
                case 2: k_red4<<<blocks, kThreads, 0, st>>>(a); break;
                default: k_red64<<<blocks, kThreads, 0, st>>>(reinterpret_cast<float4*>(a)); break;
            }
            if (e == cudaSuccess) e = cudaGetLastError();
            if (rep == 1 && e == cudaSuccess) e = cudaEventRecord(e1, st);
        }
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e == cudaSuccess) rates[k] = ms > 0.0f ? counts[k] / (ms * 1e-3) : 0.0;
    }
    if (st) cudaStreamSynchronize(st);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    cudaFree(a);
    cudaFree(sink);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? MLEM_ERR_NOMEM : MLEM_ERR_CUDA;
    }
    return MLEM_OK;
}
