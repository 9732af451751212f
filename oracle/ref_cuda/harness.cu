// harness.cu -- TEST INFRASTRUCTURE ONLY: the reference's own CUDA kernels as
// a comparison baseline on the same GPU.
//
// mlem_cuda/helper_files/cudaKernels.cu is compiled unmodified from the
// reference tree beside this file (oracle/Makefile -> oracle/_ref/
// libref_cuda.so).  ref_cuda_mlem runs the MLEM iteration of the reference's
// CUDA drivers with those kernels, one GPU, no MPI:
//   variant 4 (mlem_cuda/versions/version_4.cu:118-214): blocks of 1024,
//     d_mat_vec_mul (a thread per row), d_calcCorrel, d_tran_mat_vec_mul (a
//     thread per row, atomics), d_update; column sums by d_tran_mat_vec_mul of
//     a vector of ones (:130-132);
//   variant 6 (version_6.cu:125-212): blocks of 64, the back projection and
//     column sums by trans_mat_vec_mul_warp / trans_mat_unit_vec_mul_warp (a
//     warp per row).  Its forward projection, mat_vec_mul_warp, calls
//     __syncthreads() inside a row loop whose trip count differs between the
//     warps of a block (cudaKernels.cu:236-265) and is not run here;
//     d_mat_vec_mul stands in.
// Each iteration clears fwproj, update and correlation first, as the drivers
// do (version_4.cu:165-167).  The matrix is converted to the drivers'
// structure-of-arrays int32 CSR (helper.cu:189-208 csr_format_for_cuda), so
// nnz must stay below 2^31; the sinogram is passed as float, as the drivers
// load it.  The initial image uses seqcsr4mlem's double sums (the drivers'
// float sums differ in the last bits).  Per-kernel device times come from
// CUDA events around every launch, averaged over the timed iterations.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>
#include <vector>

#include "cudaKernels.cuh"

namespace {

struct Ev {
    cudaEvent_t a = nullptr, b = nullptr;
    Ev() { cudaEventCreate(&a); cudaEventCreate(&b); }
    ~Ev() { cudaEventDestroy(a); cudaEventDestroy(b); }
};

}  // namespace

extern "C" {

// times[5]: mean ms per iteration of clear (3 memsets), forward projection,
// correlation, back projection, update; times[5] = whole iteration.
// Returns 0, -1 for a bad argument / too many elements, -2 for a CUDA error.
int ref_cuda_mlem(const uint64_t* row_end, const void* elems, uint32_t R, uint32_t C,
                  const int32_t* sino, int n_iter, int variant, float* image_out,
                  double* times) {
    if (!row_end || !sino || !image_out || R == 0 || C == 0 || n_iter < 0) return -1;
    if (variant != 4 && variant != 6) return -1;
    const uint64_t Z = row_end[R - 1];
    if (Z >= (1ull << 31)) return -1;
    // structure-of-arrays int32 CSR, float sinogram
    std::vector<int> rowind((size_t)R + 1), colind(Z);
    std::vector<float> val(Z), lmsino(R);
    rowind[0] = 0;
    for (uint32_t r = 0; r < R; ++r) rowind[r + 1] = (int)row_end[r];
    const uint32_t* w = static_cast<const uint32_t*>(elems);
    for (uint64_t k = 0; k < Z; ++k) {
        colind[k] = (int)w[2 * k];
        std::memcpy(&val[k], &w[2 * k + 1], 4);
    }
    double sumin = 0.0;
    for (uint32_t r = 0; r < R; ++r) { lmsino[r] = (float)sino[r]; sumin += sino[r]; }

    int *rowind_d = nullptr, *colind_d = nullptr;
    float *val_d = nullptr, *lmsino_d = nullptr, *fwproj_d = nullptr, *corr_d = nullptr;
    float *update_d = nullptr, *norm_d = nullptr, *image_d = nullptr, *ones_d = nullptr;
    int rc = 0;
    auto ok = [&](cudaError_t e) { if (e != cudaSuccess && rc == 0) rc = -2; return rc == 0; };
    ok(cudaMalloc(&rowind_d, rowind.size() * 4));
    ok(cudaMalloc(&colind_d, (Z ? Z : 1) * 4));
    ok(cudaMalloc(&val_d, (Z ? Z : 1) * 4));
    ok(cudaMalloc(&lmsino_d, (size_t)R * 4));
    ok(cudaMalloc(&fwproj_d, (size_t)R * 4));
    ok(cudaMalloc(&corr_d, (size_t)R * 4));
    ok(cudaMalloc(&ones_d, (size_t)R * 4));
    ok(cudaMalloc(&update_d, (size_t)C * 4));
    ok(cudaMalloc(&norm_d, (size_t)C * 4));
    ok(cudaMalloc(&image_d, (size_t)C * 4));
    if (rc == 0) {
        ok(cudaMemcpy(rowind_d, rowind.data(), rowind.size() * 4, cudaMemcpyHostToDevice));
        if (Z) ok(cudaMemcpy(colind_d, colind.data(), Z * 4, cudaMemcpyHostToDevice));
        if (Z) ok(cudaMemcpy(val_d, val.data(), Z * 4, cudaMemcpyHostToDevice));
        ok(cudaMemcpy(lmsino_d, lmsino.data(), (size_t)R * 4, cudaMemcpyHostToDevice));
    }
    const dim3 block(variant == 4 ? 1024 : 64);
    const dim3 grid((unsigned)(((R > C ? R : C) + block.x - 1) / block.x));
    // column sums (version_4.cu:130-132, version_6.cu:139)
    if (rc == 0) {
        ok(cudaMemset(norm_d, 0, (size_t)C * 4));
        d_set_value<<<grid, block>>>(ones_d, 1.0f, R);
        if (variant == 4)
            d_tran_mat_vec_mul<<<grid, block>>>(norm_d, ones_d, val_d, rowind_d, colind_d, R);
        else
            trans_mat_unit_vec_mul_warp<<<grid, block>>>(0, R, rowind_d, colind_d, val_d, norm_d);
        ok(cudaGetLastError());
        ok(cudaDeviceSynchronize());
    }
    if (rc == 0) {
        std::vector<float> norm(C);
        ok(cudaMemcpy(norm.data(), norm_d, (size_t)C * 4, cudaMemcpyDeviceToHost));
        double sumnorm = 0.0;
        for (uint32_t i = 0; i < C; ++i) sumnorm += norm[i];
        const float initial = (float)(sumin / sumnorm);
        d_set_value<<<grid, block>>>(image_d, initial, C);
        ok(cudaGetLastError());
    }
    double acc[6] = {0, 0, 0, 0, 0, 0};
    {
        Ev e[6];
        for (int it = 0; it < n_iter && rc == 0; ++it) {
            ok(cudaEventRecord(e[0].a));
            ok(cudaMemset(fwproj_d, 0, (size_t)R * 4));
            ok(cudaMemset(update_d, 0, (size_t)C * 4));
            ok(cudaMemset(corr_d, 0, (size_t)R * 4));
            ok(cudaEventRecord(e[0].b));
            ok(cudaEventRecord(e[1].a));
            d_mat_vec_mul<<<grid, block>>>(fwproj_d, image_d, val_d, rowind_d, colind_d, R);
            ok(cudaEventRecord(e[1].b));
            ok(cudaEventRecord(e[2].a));
            d_calcCorrel<<<grid, block>>>(fwproj_d, lmsino_d, corr_d, R);
            ok(cudaEventRecord(e[2].b));
            ok(cudaEventRecord(e[3].a));
            if (variant == 4)
                d_tran_mat_vec_mul<<<grid, block>>>(update_d, corr_d, val_d, rowind_d, colind_d, R);
            else
                trans_mat_vec_mul_warp<<<grid, block>>>(0, R, rowind_d, colind_d, val_d, corr_d,
                                                        update_d);
            ok(cudaEventRecord(e[3].b));
            ok(cudaEventRecord(e[4].a));
            d_update<<<grid, block>>>(update_d, norm_d, image_d, (int)C);
            ok(cudaEventRecord(e[4].b));
            ok(cudaGetLastError());
            ok(cudaEventSynchronize(e[4].b));
            if (it == 0 && n_iter > 1) continue;  // first iteration: warm-up, not timed
            for (int p = 0; p < 5; ++p) {
                float ms = 0.0f;
                ok(cudaEventElapsedTime(&ms, e[p].a, e[p].b));
                acc[p] += ms;
            }
            float whole = 0.0f;
            ok(cudaEventElapsedTime(&whole, e[0].a, e[4].b));
            acc[5] += whole;
        }
    }
    const int timed = n_iter > 1 ? n_iter - 1 : n_iter;
    if (times)
        for (int p = 0; p < 6; ++p) times[p] = timed > 0 ? acc[p] / timed : 0.0;
    if (rc == 0) ok(cudaMemcpy(image_out, image_d, (size_t)C * 4, cudaMemcpyDeviceToHost));
    for (void* p : {(void*)rowind_d, (void*)colind_d, (void*)val_d, (void*)lmsino_d,
                    (void*)fwproj_d, (void*)corr_d, (void*)ones_d, (void*)update_d,
                    (void*)norm_d, (void*)image_d})
        if (p) cudaFree(p);
    return rc;
}

}  // extern "C"
