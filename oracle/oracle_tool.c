/*
 * oracle_tool.c -- command-line front end of the oracle (TEST INFRASTRUCTURE).
 *
 * Runs the checker and the synthetic-input generator as a separate process, so
 * that a benchmark can run them on host cores beside the GPU work, and so that
 * the process which times the reference's own binaries loads no library of the
 * package under test.
 *
 *   oracle_tool f64-mlem MATRIX.csr4 SINO.i32 ITERS THREADS OUT.f64
 *       FP64 MLEM (oracle_mlem_f64_threads: the iteration of
 *       mlem_seq/seqcsr4mlem.cpp:137-189 with every quantity in double);
 *       writes the double image.
 *   oracle_tool synth-matrix NX NY NZ ROWS MIN MAX SEED RADIUS_SCALE MIN_LEN OUT.csr4
 *       The seeded Siddon matrix of the synthetic workloads (the generator of
 *       mlem_b200/gen/siddon_core.h, compiled into this tool) as a CSR4 file
 *       with the minimal 60-byte scanner block carrying the voxel grid.
 *   oracle_tool project-f64 MATRIX.csr4 X.f32 OUT.f64
 *       Sequential double projection out = A x (the sinogram means).
 *
 * The CSR4 layout is that of helper_files_common/csr4matrix.cpp:32-157: a
 * 28-byte header (b"PCSR", version 4, flags, nRows u32 @8, nColumns u32 @12,
 * nnz u64 @16, scanConfigBytes u32 @24), the scanner block, nRows uint64 row
 * END offsets, then nnz 8-byte {uint32 column, float32 value} elements.
 */
#define _GNU_SOURCE
#include <errno.h>
#include <fcntl.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include "mlem_oracle.h"

uint64_t mlem_gen_siddon_counts(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t R,
                                uint32_t min_count, uint32_t max_count, double radius_scale,
                                double min_len, uint64_t seed, uint32_t* counts);
int mlem_gen_siddon_fill(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t R, uint32_t min_count,
                         uint32_t max_count, double radius_scale, double min_len, uint64_t seed,
                         const uint64_t* row_end, void* elems);

typedef struct {
    uint32_t R, C;
    uint64_t nnz;
    const uint64_t* row_end;
    const oracle_elem* elems;
    void* map;
    size_t map_len;
} csr4_file;

static int die(const char* msg, const char* arg) {
    fprintf(stderr, "oracle_tool: %s%s%s\n", msg, arg ? " " : "", arg ? arg : "");
    return 1;
}

static uint32_t rd32(const unsigned char* p) {
    uint32_t v;
    memcpy(&v, p, 4);
    return v;
}

static uint64_t rd64(const unsigned char* p) {
    uint64_t v;
    memcpy(&v, p, 8);
    return v;
}

static int open_csr4(const char* path, csr4_file* m) {
    int fd = open(path, O_RDONLY);
    if (fd < 0) return die("cannot open", path);
    struct stat st;
    if (fstat(fd, &st) != 0 || st.st_size < 28) {
        close(fd);
        return die("too short:", path);
    }
    void* map = mmap(NULL, (size_t)st.st_size, PROT_READ, MAP_SHARED, fd, 0);
    close(fd);
    if (map == MAP_FAILED) return die("mmap failed:", path);
    const unsigned char* h = (const unsigned char*)map;
    if (memcmp(h, "PCSR", 4) != 0 || h[4] != 4) {
        munmap(map, (size_t)st.st_size);
        return die("not a CSR4 (version 4) file:", path);
    }
    m->R = rd32(h + 8);
    m->C = rd32(h + 12);
    m->nnz = rd64(h + 16);
    const uint64_t off = 28 + (uint64_t)rd32(h + 24);
    const uint64_t need = off + 8ull * m->R + 8ull * m->nnz;
    if ((uint64_t)st.st_size < need || off % 8 != 0) {
        munmap(map, (size_t)st.st_size);
        return die("size or alignment does not match the header:", path);
    }
    m->row_end = (const uint64_t*)(h + off);
    m->elems = (const oracle_elem*)(h + off + 8ull * m->R);
    if (m->R && m->row_end[m->R - 1] != m->nnz) {
        munmap(map, (size_t)st.st_size);
        return die("last row END offset differs from nnz:", path);
    }
    for (uint32_t r = 1; r < m->R; ++r)
        if (m->row_end[r] < m->row_end[r - 1]) {
            munmap(map, (size_t)st.st_size);
            return die("row END offsets decrease:", path);
        }
    for (uint64_t k = 0; k < m->nnz; ++k)
        if (m->elems[k].index >= m->C) {
            munmap(map, (size_t)st.st_size);
            return die("column index out of range:", path);
        }
    m->map = map;
    m->map_len = (size_t)st.st_size;
    return 0;
}

static void* read_all(const char* path, size_t* len) {
    FILE* f = fopen(path, "rb");
    if (!f) return NULL;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    void* buf = malloc(n > 0 ? (size_t)n : 1);
    if (buf && n > 0 && fread(buf, 1, (size_t)n, f) != (size_t)n) {
        free(buf);
        buf = NULL;
    }
    fclose(f);
    *len = n > 0 ? (size_t)n : 0;
    return buf;
}

static int write_all(const char* path, const void* p, size_t n) {
    FILE* f = fopen(path, "wb");
    if (!f) return die("cannot write", path);
    int ok = fwrite(p, 1, n, f) == n;
    ok &= fclose(f) == 0;
    return ok ? 0 : die("write failed:", path);
}

static int cmd_f64_mlem(int argc, char** argv) {
    if (argc != 7) return die("usage: f64-mlem MATRIX SINO ITERS THREADS OUT", NULL);
    csr4_file m;
    if (open_csr4(argv[2], &m)) return 1;
    size_t slen = 0;
    int32_t* sino = (int32_t*)read_all(argv[3], &slen);
    if (!sino || slen != 4ull * m.R) return die("sinogram length differs from the row count:", argv[3]);
    const int iters = atoi(argv[4]), threads = atoi(argv[5]);
    double* img = (double*)malloc((size_t)m.C * sizeof(double) + 1);
    if (!img) return die("out of memory", NULL);
    int rc = oracle_mlem_f64_threads(m.R, m.C, m.row_end, m.elems, sino, m.R, iters, threads, img);
    if (rc != 0) return die("oracle_mlem_f64_threads failed", NULL);
    rc = write_all(argv[6], img, (size_t)m.C * sizeof(double));
    free(img);
    free(sino);
    munmap(m.map, m.map_len);
    return rc;
}

static int cmd_synth_matrix(int argc, char** argv) {
    if (argc != 12)
        return die("usage: synth-matrix NX NY NZ ROWS MIN MAX SEED RADIUS_SCALE MIN_LEN OUT", NULL);
    const uint32_t nx = (uint32_t)strtoul(argv[2], NULL, 10), ny = (uint32_t)strtoul(argv[3], NULL, 10),
                   nz = (uint32_t)strtoul(argv[4], NULL, 10), R = (uint32_t)strtoul(argv[5], NULL, 10),
                   lo = (uint32_t)strtoul(argv[6], NULL, 10), hi = (uint32_t)strtoul(argv[7], NULL, 10);
    const uint64_t seed = strtoull(argv[8], NULL, 10);
    const double rs = strtod(argv[9], NULL), ml = strtod(argv[10], NULL);
    const uint64_t C = (uint64_t)nx * ny * nz;
    if (C == 0 || C > 0xFFFFFFFFull) return die("bad grid", NULL);
    uint32_t* counts = (uint32_t*)malloc((size_t)R * sizeof(uint32_t) + 1);
    uint64_t* row_end = (uint64_t*)malloc((size_t)R * sizeof(uint64_t) + 1);
    if (!counts || !row_end) return die("out of memory", NULL);
    const uint64_t Z = mlem_gen_siddon_counts(nx, ny, nz, R, lo, hi, rs, ml, seed, counts);
    uint64_t acc = 0;
    for (uint32_t r = 0; r < R; ++r) row_end[r] = (acc += counts[r]);
    free(counts);
    void* el = malloc((size_t)Z * 8 + 8);
    if (!el) return die("out of memory", NULL);
    if (mlem_gen_siddon_fill(nx, ny, nz, R, lo, hi, rs, ml, seed, row_end, el) != 0)
        return die("generator fill disagrees with its counts", NULL);
    /* header + the minimal scanner block: one layer (5 floats), one block of
     * size 1, one ring, voxel size 1, the grid */
    unsigned char head[28 + 60];
    memset(head, 0, sizeof head);
    memcpy(head, "PCSR", 4);
    head[4] = 4;
    const uint32_t Cu = (uint32_t)C, scb = 60;
    memcpy(head + 8, &R, 4);
    memcpy(head + 12, &Cu, 4);
    memcpy(head + 16, &Z, 8);
    memcpy(head + 24, &scb, 4);
    unsigned char* s = head + 28;
    const uint32_t one = 1;
    const float lay[5] = {1.0f, 1.0f, 1.0f, 1.0f, 0.0f}, vs[3] = {1.0f, 1.0f, 1.0f};
    const uint32_t grid[3] = {nx, ny, nz};
    memcpy(s, &one, 4);
    memcpy(s + 4, lay, 20);
    memcpy(s + 24, &one, 4);  /* n_blocks */
    memcpy(s + 28, &one, 4);  /* block_size (no gaps) */
    memcpy(s + 32, &one, 4);  /* n_rings (no gaps) */
    memcpy(s + 36, vs, 12);
    memcpy(s + 48, grid, 12);
    FILE* f = fopen(argv[11], "wb");
    if (!f) return die("cannot write", argv[11]);
    int ok = fwrite(head, 1, sizeof head, f) == sizeof head;
    ok &= fwrite(row_end, 8, R, f) == R;
    ok &= fwrite(el, 8, (size_t)Z, f) == (size_t)Z;
    ok &= fclose(f) == 0;
    free(el);
    free(row_end);
    return ok ? 0 : die("write failed:", argv[11]);
}

static int cmd_project_f64(int argc, char** argv) {
    if (argc != 5) return die("usage: project-f64 MATRIX X.f32 OUT.f64", NULL);
    csr4_file m;
    if (open_csr4(argv[2], &m)) return 1;
    size_t xlen = 0;
    float* x = (float*)read_all(argv[3], &xlen);
    if (!x || xlen != 4ull * m.C) return die("image length differs from the column count:", argv[3]);
    double* out = (double*)malloc((size_t)m.R * sizeof(double) + 1);
    if (!out) return die("out of memory", NULL);
    oracle_project_f64(m.R, m.row_end, m.elems, x, out);
    int rc = write_all(argv[4], out, (size_t)m.R * sizeof(double));
    free(out);
    free(x);
    munmap(m.map, m.map_len);
    return rc;
}

int main(int argc, char** argv) {
    if (argc < 2) return die("usage: oracle_tool f64-mlem|synth-matrix|project-f64 ...", NULL);
    if (!strcmp(argv[1], "f64-mlem")) return cmd_f64_mlem(argc, argv);
    if (!strcmp(argv[1], "synth-matrix")) return cmd_synth_matrix(argc, argv);
    if (!strcmp(argv[1], "project-f64")) return cmd_project_f64(argc, argv);
    return die("unknown command", argv[1]);
}
