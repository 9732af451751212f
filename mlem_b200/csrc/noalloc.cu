// noalloc.cu -- one MLEM iteration that allocates no device memory.
//
// Every other entry point keeps its working vectors in memory the library
// allocates with cudaMalloc.  Some callers cannot allow that: a host program
// that runs under a fixed, pre-reserved device-memory budget (a memory pool
// handed to it by a framework or a scheduler), or code that runs while
// another component owns the device allocator.  mlem_iterate_noalloc_d
// serves them: the caller passes every input and output as device pointers,
// and the only working vector, the back-projection update, lives in the
// file-scope array below.
//
// The array is a fixed MLEM_NOALLOC_MAX_VOXELS floats (4 MiB).  Every GPU
// that loads this library holds it until the process exits, whether or not
// the entry point is ever called.  All calls on a device share it, and it
// keeps the last call's contents, so each call clears the part it uses
// before use, and calls that overlap on the GPU (two streams, two host
// threads) race on it.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"
#include "mlem_b200.h"
#include "host/errors.hpp"

using namespace mlem;

namespace {

static __device__ __align__(256) float g_update_scratch[MLEM_NOALLOC_MAX_VOXELS];
// bit 0: a column index >= n_cols; bit 1: a row whose offsets decrease or
// pass the element count
static __device__ unsigned int g_bad_input;

constexpr unsigned int kBadColumn = 1u, kBadOffsets = 2u;

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
struct DeviceScratch {
    unsigned long long ctx_id;  // the context the addresses belong to
    float* update;
    unsigned int* flag;
};
DeviceScratch g_scratch[kMaxDevices] = {};

// One pass per row: forward projection, calcCorrel, and the scatter of the
// row into the update vector (the one-pass method of k_project.cu, here with
// bounds checks on every row's offsets and every column instead of an
// up-front validation pass, which would need memory).  A warp per row; all
// lanes of a warp read the same offsets, so a row that fails its check is
// skipped by the whole warp.  8-byte element loads.
__global__ void __launch_bounds__(256) k_noalloc_row(const uint64_t* __restrict__ row_ptr,
                                                     const uint2* __restrict__ el, uint64_t n_elems,
                                                     uint32_t R, uint32_t C,
                                                     const float* __restrict__ x,
                                                     const int32_t* __restrict__ sino,
                                                     float* __restrict__ u,
                                                     unsigned int* __restrict__ bad) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t r = warp; r < R; r += nwarps) {
        const uint64_t b = row_ptr[r], e = row_ptr[r + 1];
        if (b > e || e > n_elems) {
            if (lane == 0) atomicOr(bad, kBadOffsets);
            continue;
        }
        float acc = 0.0f;
        for (uint64_t k = b + lane; k < e; k += 32) {
            const uint2 q = el[k];
            if (q.x < C) acc = fmaf(__uint_as_float(q.y), x[q.x], acc);
            else atomicOr(bad, kBadColumn);
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

// Identity of the context current on this thread (0 if none is current yet),
// from the driver's cuCtxGetCurrent / cuCtxGetId, reached through the
// runtime's entry-point query so the library needs no link to libcuda.
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
        looked_up = true;
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device addresses of the scratch array and the flag.  In host code the names
// g_update_scratch / g_bad_input are only host-side handles, not device
// addresses: a kernel must be given the looked-up pointers.  They are looked
// up with the device current, once per device and context: a context
// created again (after cudaDeviceReset, say) loads the module again, and its
// addresses may differ, so they are looked up again.
int device_scratch(int dev, float** scratch, unsigned int** flag) {
    if (dev < 0 || dev >= kMaxDevices)
        return set_error(nullptr, MLEM_ERR_INVALID, "device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceScratch& d = g_scratch[dev];
    unsigned long long id = current_context_id();
    if (!d.update || id == 0 || id != d.ctx_id) {
        void* s = nullptr;
        void* f = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&s, g_update_scratch);
        if (e == cudaSuccess) e = cudaGetSymbolAddress(&f, g_bad_input);
        if (e != cudaSuccess)
            return set_error(nullptr, MLEM_ERR_CUDA, "cudaGetSymbolAddress: %s",
                             cudaGetErrorString(e));
        d.update = static_cast<float*>(s);
        d.flag = static_cast<unsigned int*>(f);
        d.ctx_id = id ? id : current_context_id();  // the lookup made the context current
    }
    *scratch = d.update;
    *flag = d.flag;
    return MLEM_OK;
}

}  // namespace

extern "C" int mlem_iterate_noalloc_d(const uint64_t* row_ptr, const void* elems, uint64_t n_elems,
                                      uint32_t n_rows, uint32_t n_cols, const int32_t* sino,
                                      const float* norm, float* image, void* stream) {
    if (n_cols > MLEM_NOALLOC_MAX_VOXELS)
        return set_error(nullptr, MLEM_ERR_INVALID,
                         "mlem_iterate_noalloc_d: %u voxels exceed the fixed scratch of %d voxels; "
                         "use a context (mlem_create) for larger images",
                         n_cols, MLEM_NOALLOC_MAX_VOXELS);
    if (!row_ptr || !sino || !norm || !image || (n_elems && !elems))
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
                                                     n_elems, n_rows, n_cols, image, sino, u, bad);
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
    if (hbad & kBadOffsets)
        return set_error(nullptr, MLEM_ERR_MATRIX,
                         "mlem_iterate_noalloc_d: a row's offsets decrease or pass n_elems (those "
                         "rows were skipped)%s",
                         (hbad & kBadColumn) ? "; a column index is >= n_cols (skipped)" : "");
    if (hbad & kBadColumn)
        return set_error(nullptr, MLEM_ERR_MATRIX,
                         "mlem_iterate_noalloc_d: a column index is >= n_cols (those elements "
                         "were skipped)");
    return MLEM_OK;
}
