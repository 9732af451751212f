// main.cpp -- mlem_b200: drop-in for the reference's seqcsr4mlem / openmpcsr4mlem.
//
//   mlem_b200 <matrix> <input> <output> <iterations> [<checkpointing>]
//
// Same positional arguments (mlem_seq/seqcsr4mlem.cpp:22-34), plus the
// optional fifth argument of the MPI/CUDA drivers (mlem_mpi/mpicsr4mlem.cpp
// :163-175): a checkpoint interval.  With it, the driver restores from
// img.chkpt + iter.chkpt in the working directory when both exist
// (mpicsr4mlem.cpp:536-553), writes both every `checkpointing` iterations
// ((iter+1) % checkpointing == 0, mlem_cuda/helper_files/hybCalcFunc.cu
// :852-853) and removes them after a normal exit when checkpointing > 0
// (hybCalcFunc.cu:895-902).  Files: CSR4 matrix, int32 sinogram, float32
// image (helper_files_common/csr4matrix.cpp, vector.hpp).
//
// Batched extension: <input> and <output> may be comma-separated lists of
// equal length; the B sinograms are then reconstructed together in one pass
// over the matrix per iteration.  Checkpoints are single-frame only.
//
// Environment: MLEM_B200_DEVICE (GPU index, default 0), MLEM_B200_EXACT=1
// (bit-exact kernels), MLEM_B200_AUTOTUNE=1 (tune the kernels for this
// matrix before iterating; deterministic CSC back projection unless
// MLEM_B200_AUTOTUNE=any), MLEM_B200_CSV=1 (print "iter,elapsed" lines like
// openmpcsr4mlem built with -DMESSUNG, openmpcsr4mlem.cpp:217),
// MLEM_B200_EXPAND_SYMMETRY=1 (reconstruct with the full matrix of a
// symmetry-compressed file; by default its symmetry flags are ignored, as the
// reference's drivers ignore them; =kernels: the same reconstruction with only
// the stored elements on the GPU and the mirrors applied in the kernels),
// MLEM_B200_TIMING=1 (the elapsed time after each phase -- matrix, sinograms,
// tuning, iterations, output -- as "phase,<name>,<seconds>" lines on stderr).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "mlem_b200.h"

namespace {

struct Options {
    std::string matrix;
    std::vector<std::string> inputs, outputs;
    int iterations = 0;
    bool has_checkpointing = false;
    int checkpointing = 0;
};

std::vector<std::string> split(const std::string& s) {
    std::vector<std::string> out;
    std::stringstream ss(s);
    std::string item;
    while (std::getline(ss, item, ',')) out.push_back(item);
    return out;
}

int parse_int(const char* s, const char* what) {
    try {
        size_t pos = 0;
        int v = std::stoi(s, &pos);
        if (pos != std::strlen(s)) throw std::invalid_argument(s);
        return v;
    } catch (const std::exception&) {
        throw std::runtime_error(std::string("invalid ") + what + ": " + s);
    }
}

Options parse(int argc, char** argv) {
    if (argc != 5 && argc != 6) throw std::runtime_error("wrong number of command line parameters");
    Options o;
    o.matrix = argv[1];
    o.inputs = split(argv[2]);
    o.outputs = split(argv[3]);
    o.iterations = parse_int(argv[4], "iterations");
    if (argc == 6) {
        o.has_checkpointing = true;
        o.checkpointing = parse_int(argv[5], "checkpointing");
    }
    if (o.inputs.empty() || o.inputs.size() != o.outputs.size())
        throw std::runtime_error("input and output lists must have the same length");
    if (o.iterations < 0) throw std::runtime_error("iterations must be >= 0");
    if (o.inputs.size() > 1 && o.has_checkpointing && o.checkpointing > 0)
        throw std::runtime_error("checkpointing is supported for a single sinogram only");
    return o;
}

void check(int status, mlem_ctx* ctx) {
    if (status != MLEM_OK) {
        std::string msg = ctx ? mlem_last_error(ctx) : mlem_global_error();
        throw std::runtime_error(std::string(mlem_status_string(status)) + ": " + msg);
    }
}

int env_int(const char* name, int dflt) {
    const char* v = std::getenv(name);
    return (v && *v) ? std::atoi(v) : dflt;
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

int run(int argc, char** argv) {
    Options o = parse(argc, argv);
    const bool csv = env_int("MLEM_B200_CSV", 0) != 0;
    if (!csv) {
        std::cout << "Matrix file: " << o.matrix << std::endl;
        std::cout << "Input file: " << argv[2] << std::endl;
        std::cout << "Output file: " << argv[3] << std::endl;
        std::cout << "Iterations: " << o.iterations << std::endl;
        if (o.has_checkpointing) std::cout << "Checkpointing: " << o.checkpointing << std::endl;
    }
    uint32_t flags = env_int("MLEM_B200_EXACT", 0) ? MLEM_FLAG_EXACT : 0u;
    const char* expand = std::getenv("MLEM_B200_EXPAND_SYMMETRY");
    if (expand && std::strcmp(expand, "kernels") == 0) flags |= MLEM_FLAG_MIRROR_KERNELS;
    else if (env_int("MLEM_B200_EXPAND_SYMMETRY", 0)) flags |= MLEM_FLAG_EXPAND_SYMMETRY;
    const int device = env_int("MLEM_B200_DEVICE", 0);

    auto t0 = std::chrono::steady_clock::now();
    // MLEM_B200_TIMING=1: "phase,<name>,<seconds since the matrix load began>" on stderr
    const bool timing = env_int("MLEM_B200_TIMING", 0) != 0;
    auto phase = [&](const char* name) {
        if (timing) std::cerr << "phase," << name << "," << seconds_since(t0) << std::endl;
    };
    mlem_ctx* ctx = nullptr;
    check(mlem_create_from_file(&ctx, o.matrix.c_str(), flags, device), nullptr);
    phase("matrix");
    struct Guard { mlem_ctx* c; ~Guard() { mlem_destroy(c); } } guard{ctx};
    mlem_info info;
    check(mlem_get_info(ctx, &info), ctx);
    if (!csv)
        std::cout << "Calculated norm, elapsed time: " << seconds_since(t0) << "s\n";

    const uint32_t B = (uint32_t)o.inputs.size();
    const uint32_t R = info.n_rows, C = info.n_cols;
    std::vector<int32_t> sino((size_t)B * R);
    for (uint32_t b = 0; b < B; ++b) {
        uint64_t n = 0;
        check(mlem_vector_read(o.inputs[b].c_str(), 4, nullptr, 0, &n), nullptr);
        if (n != R) {  // the reference asserts this in calcCorrel (seqcsr4mlem.cpp:96)
            std::ostringstream ss;
            ss << "sinogram " << o.inputs[b] << " has " << n << " entries, the matrix " << R << " rows";
            throw std::runtime_error(ss.str());
        }
        check(mlem_vector_read(o.inputs[b].c_str(), 4, sino.data() + (size_t)b * R, R, &n), nullptr);
    }
    check(mlem_set_sinograms(ctx, sino.data(), B), ctx);
    phase("sinograms");

    int first = 0;
    std::vector<float> image((size_t)C * B);
    bool restored = false;
    if (o.has_checkpointing && B == 1) {
        int32_t next = 0;
        const int s = mlem_checkpoint_read(".", image.data(), C, &next);
        if (s == MLEM_OK) {
            check(mlem_set_images(ctx, image.data()), ctx);
            first = next;
            restored = true;
            if (!csv) std::cout << "I got Checkpoint at iteration " << first << "\n";
        } else if (s != MLEM_NO_CHECKPOINT) {
            check(s, nullptr);
        } else if (!csv && std::strcmp(mlem_global_error(), "omitted incomplete checkpoint") == 0) {
            std::cout << "omitted incomplete checkpoint\n";
        }
    }
    if (!restored) {
        std::vector<float> init(B);
        check(mlem_init_images(ctx, init.data()), ctx);
        if (!csv)
            for (uint32_t b = 0; b < B; ++b) {
                float v = 0;
                check(mlem_init_value(ctx, sino.data() + (size_t)b * R, R, &v), ctx);
                std::cout << "INIT: initial value=" << v << std::endl;
            }
    }
    const char* tune = std::getenv("MLEM_B200_AUTOTUNE");
    const bool autotune = tune && *tune && std::strcmp(tune, "0") != 0;
    if (!autotune && info.has_csc && !(info.flags & (MLEM_FLAG_EXACT | MLEM_FLAG_MIRROR_KERNELS))) {
        // The default method stays the deterministic CSC back projection; with
        // the row order it walks the CSC in visiting order (a second CSC,
        // built here), whose gathers fall on neighbouring rays.  Without the
        // row order or the memory for it, the file-order CSC runs.
        mlem_tuning t;
        check(mlem_get_tuning(ctx, &t), ctx);
        t.bk_mode = MLEM_BK_CSC;
        t.group = 32;
        t.blocks_per_sm = 8;  // the forward pass (plain-full: 1.52 ms against 1.55-1.59 at 4)
        t.visit = MLEM_VISIT_SORTED;
        if (mlem_set_tuning(ctx, &t) != MLEM_OK && !csv)
            std::cout << "CSC in visiting order unavailable (" << mlem_last_error(ctx)
                      << "); file-order CSC\n";
    }
    if (autotune) {
        mlem_tuning t;
        // the mirrored kernels have atomics only: no deterministic choice to restrict to
        const bool any = std::strcmp(tune, "any") == 0 || (info.flags & MLEM_FLAG_MIRROR_KERNELS);
        check(mlem_autotune(ctx, any ? 0 : 1, &t), ctx);
        if (!csv)
            std::cout << "Autotuned: mode " << t.bk_mode << ", group " << t.group << ", frame tile "
                      << t.frame_tile << ", row visit " << t.visit << ", " << t.ms_per_iter
                      << " ms/iteration\n";
    }
    phase("tuning");
    if (!csv) std::cout << "Starting " << (o.iterations - first) << " MLEM iterations" << std::endl;

    const int chk = o.has_checkpointing ? o.checkpointing : 0;
    int iter = first;
    while (iter < o.iterations) {
        // run up to the next checkpoint boundary in one call (one graph launch)
        int stop = o.iterations;
        if (chk > 0) {
            const int next_chk = ((iter / chk) + 1) * chk;  // first (it+1) % chk == 0 boundary
            if (next_chk < stop) stop = next_chk;
        }
        const int n = stop - iter;
        std::vector<double> sums((size_t)n * B);
        std::vector<uint64_t> zeros((size_t)n * B), subn((size_t)n * B);
        auto t1 = std::chrono::steady_clock::now();
        check(mlem_iterate(ctx, n, sums.data(), zeros.data(), subn.data()), ctx);
        const double per = seconds_since(t1) / n;
        for (int k = 0; k < n; ++k) {
            const int it = iter + k;
            if (csv) {
                std::cout << it << "," << per << std::endl;
                continue;
            }
            for (uint32_t b = 0; b < B; ++b) {
                const size_t i = (size_t)k * B + b;
                std::cout << "Finished iteration " << it + 1 << ", ";
                if (B > 1) std::cout << "frame " << b << ", ";
                std::cout << " image sum: " << sums[i] << ", elapsed time: " << per << "s\n";
                std::cout << "Zeros: " << zeros[i] << " (" << (float)zeros[i] / C * 100.0 << " %), "
                          << " subnormals: " << subn[i] << " (" << (float)subn[i] / C * 100.0
                          << " %)\n";
            }
        }
        iter = stop;
        if (chk > 0 && iter % chk == 0 && iter < o.iterations) {
            check(mlem_get_images(ctx, image.data()), ctx);
            check(mlem_checkpoint_write(".", image.data(), C, iter), nullptr);
            if (!csv) std::cout << "creating checkpoint " << std::endl;
        }
    }
    phase("iterations");
    check(mlem_get_images(ctx, image.data()), ctx);
    for (uint32_t b = 0; b < B; ++b)
        check(mlem_vector_write(o.outputs[b].c_str(), image.data() + (size_t)b * C, 4, C, 0), nullptr);
    phase("output");
    if (chk > 0) mlem_checkpoint_remove(".");
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        return run(argc, argv);
    } catch (const std::exception& e) {
        std::cerr << "mlem_b200: " << e.what() << std::endl;
        return 1;
    }
}
