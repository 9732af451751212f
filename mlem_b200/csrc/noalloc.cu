// noalloc.cu -- one MLEM iteration that allocates no device memory.
//
// Every other entry point keeps its working vectors in memory the library
// allocates with cudaMalloc.  Some callers cannot allow that: a host program
// that runs under a fixed, pre-reserved device-memory budget (a memory pool
// handed to it by a framework or a scheduler), code that runs while another
// component owns the allocator, or a caller that must not add allocations to
// a captured or latency-critical section.  mlem_iterate_noalloc_d serves
// them: the caller passes every input and output as device pointers, and the
// only working vector, the back-projection update, lives in the file-scope
// array below.
//
// The array is a fixed MLEM_NOALLOC_MAX_VOXELS floats (4 MiB).  Every GPU
// that loads this library holds it until the process exits, whether or not
// the entry point is ever called.  All calls on a device share it, and it
// keeps the last call's contents, so each call clears the part it uses
// before use, and calls that overlap on the GPU (two streams, two host
// threads) race on it.
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"
#include "mlem_b200.h"
#include "host/errors.hpp"

using namespace mlem;

namespace {

__device__ __align__(256) float g_update_scratch[MLEM_NOALLOC_MAX_VOXELS];
__device__ unsigned int g_bad_column;

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
float* g_scratch_addr[kMaxDevices] = {};
unsigned int* g_flag_addr[kMaxDevices] = {};

// One pass per row: forward projection, calcCorrel, and the scatter of the
// row into the update vector (the one-pass method of k_project.cu, here with
// a bounds check on every column instead of an up-front validation pass,
// which would need memory).  A warp per row; 8-byte element loads.
__global__ void __launch_bounds__(256) k_noalloc_row(const uint64_t* __restrict__ row_ptr,
                                                     const uint2* __restrict__ el, uint32_t R,
                                                     uint32_t C, const float* __restrict__ x,
                                                     const int32_t* __restrict__ sino,
                                                     float* __restrict__ u,
                                                     unsigned int* __restrict__ bad) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t r = warp; r < R; r += nwarps) {
        const uint64_t b = row_ptr[r], e = row_ptr[r + 1];
        float acc = 0.0f;
        for (uint64_t k = b + lane; k < e; k += 32) {
            const uint2 q = el[k];
            if (q.x < C) acc = fmaf(__uint_as_float(q.y), x[q.x], acc);
            else atomicOr(bad, 1u);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(MLEM_FULL_MASK, acc, o);
        const float c = correl_of(sino[r], acc);
        if (c == 0.0f) continue;
        for (uint64_t k = b + lane; k < e; k += 32) {
            const uint2 q = el[k];
            if (q.x < C) atomicAdd(u + q.x, __uint_as_float(q.y) * c);
        }
    }
}

// calcUpdate (mlem_seq/seqcsr4mlem.cpp:123-134).
__global__ void k_noalloc_update(float* __restrict__ x, const float* __restrict__ u,
                                 const float* __restrict__ norm, uint32_t C) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < C;
         i += (uint64_t)gridDim.x * blockDim.x)
        x[i] *= update_factor(u[i], norm[i]);
}

// Device addresses of the scratch array and the flag, looked up once per
// device with that device current.  In host code the names
// g_update_scratch / g_bad_column are only host-side handles, not device
// addresses: a kernel must be given the looked-up pointers.
int device_scratch(int dev, float** scratch, unsigned int** flag) {
    if (dev < 0 || dev >= kMaxDevices)
        return set_error(nullptr, MLEM_ERR_INVALID, "device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* s = nullptr;
        void* f = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&s, g_update_scratch);
        if (e == cudaSuccess) e = cudaGetSymbolAddress(&f, g_bad_column);
        if (e != cudaSuccess)
            return set_error(nullptr, MLEM_ERR_CUDA, "cudaGetSymbolAddress: %s",
                             cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<float*>(s);
        g_flag_addr[dev] = static_cast<unsigned int*>(f);
    }
    *scratch = g_scratch_addr[dev];
    *flag = g_flag_addr[dev];
    return MLEM_OK;
}

}  // namespace

extern "C" int mlem_iterate_noalloc_d(const uint64_t* row_ptr, const void* elems, uint32_t n_rows,
                                      uint32_t n_cols, const int32_t* sino, const float* norm,
                                      float* image, void* stream) {
    if (n_cols > MLEM_NOALLOC_MAX_VOXELS)
        return set_error(nullptr, MLEM_ERR_INVALID,
                         "mlem_iterate_noalloc_d: %u voxels exceed the fixed scratch of %d voxels; "
                         "use a context (mlem_create) for larger images",
                         n_cols, MLEM_NOALLOC_MAX_VOXELS);
    if (!row_ptr || !sino || !norm || !image || (n_rows && !elems))
        return set_error(nullptr, MLEM_ERR_INVALID, "mlem_iterate_noalloc_d: null pointer");
    if (n_cols == 0) return MLEM_OK;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return set_error(nullptr, MLEM_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    float* u = nullptr;
    unsigned int* bad = nullptr;
    int s = device_scratch(dev, &u, &bad);
    if (s != MLEM_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // The shared scratch keeps the previous call's contents: clear what this call uses.
    e = cudaMemsetAsync(u, 0, (size_t)n_cols * sizeof(float), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(unsigned int), st);
    if (e == cudaSuccess && n_rows) {
        k_noalloc_row<<<kB200SMs * 8, 256, 0, st>>>(row_ptr, static_cast<const uint2*>(elems),
                                                     n_rows, n_cols, image, sino, u, bad);
        e = cudaGetLastError();
    }
    unsigned int hbad = 0;
    if (e == cudaSuccess) {
        k_noalloc_update<<<kB200SMs * 4, 256, 0, st>>>(image, u, norm, n_cols);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, bad, sizeof(hbad), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return set_error(nullptr, MLEM_ERR_CUDA, "mlem_iterate_noalloc_d: %s", cudaGetErrorString(e));
    if (hbad)
        return set_error(nullptr, MLEM_ERR_MATRIX,
                         "mlem_iterate_noalloc_d: a column index is >= n_cols (those elements "
                         "were skipped)");
    return MLEM_OK;
}
