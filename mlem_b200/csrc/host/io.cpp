// io.cpp -- host side of the C ABI: the reference's file formats.
//
// CSR4 matrix (helper_files_common/csr4matrix.cpp:32-224), raw vectors
// (helper_files_common/vector.hpp:33-140), the img.chkpt / iter.chkpt pair
// (mlem_mpi/mpicsr4mlem.cpp:95-154) and the nnz-balanced row partition
// (mlem_mpi/mpicsr4mlem.cpp:202-234).  Plain POSIX IO; no CUDA.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cerrno>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "errors.hpp"
#include "mlem_b200.h"

namespace mlem {

std::string& global_error() {
    static thread_local std::string msg;
    return msg;
}

int set_error(std::string* slot, int status, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (slot) *slot = buf;
    global_error() = buf;
    return status;
}

namespace {

constexpr uint32_t kHeaderBytes = 28;      // csr4matrix.hpp:178 minHeaderLength
constexpr uint32_t kMinScanConfig = 60;    // csr4matrix.hpp:179 minScanConfigBytes
constexpr size_t kHeaderRead = 1000;       // csr4matrix.cpp:51

int err(int status, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int err(int status, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return set_error(nullptr, status, "%s", buf);
}

template <typename T>
T rd(const unsigned char* p) {
    T v;
    std::memcpy(&v, p, sizeof(T));
    return v;
}

struct Fd {
    int fd = -1;
    ~Fd() { if (fd >= 0) ::close(fd); }
};

bool read_full(int fd, void* buf, size_t n, off_t off) {
    char* p = static_cast<char*>(buf);
    while (n) {
        ssize_t k = ::pread(fd, p, n, off);
        if (k <= 0) return false;
        p += k;
        n -= (size_t)k;
        off += k;
    }
    return true;
}

bool write_full(int fd, const void* buf, size_t n) {
    const char* p = static_cast<const char*>(buf);
    while (n) {
        ssize_t k = ::write(fd, p, n);
        if (k <= 0) return false;
        p += k;
        n -= (size_t)k;
    }
    return true;
}

int parse_header(const char* path, int fd, mlem_csr4_header* h) {
    struct stat st;
    if (::fstat(fd, &st) != 0) return err(MLEM_ERR_IO, "Cannot stat file %s", path);
    const uint64_t size = (uint64_t)st.st_size;
    if (size < kHeaderBytes) return err(MLEM_ERR_FORMAT, "File too short %s", path);
    unsigned char head[kHeaderRead];
    const size_t hl = size < kHeaderRead ? (size_t)size : kHeaderRead;
    if (!read_full(fd, head, hl, 0)) return err(MLEM_ERR_IO, "Cannot read header %s", path);
    if (std::memcmp(head, "PCSR", 4) != 0)
        return err(MLEM_ERR_FORMAT, "Input file '%s' is not a CSR matrix", path);
    if (head[4] != 4)
        return err(MLEM_ERR_FORMAT, "Input file '%s' has wrong CSR version (need v4)", path);
    std::memset(h, 0, sizeof(*h));
    h->version = head[4];
    h->flags = head[5];
    h->n_rows = rd<uint32_t>(head + 8);
    h->n_cols = rd<uint32_t>(head + 12);
    h->nnz = rd<uint64_t>(head + 16);
    h->scan_config_bytes = rd<uint32_t>(head + 24);
    h->file_size = size;
    // 64-bit arithmetic (the reference's uint32 total wraps above 4 GiB, csr4matrix.cpp:85)
    if (h->nnz > (UINT64_MAX - kHeaderBytes) / 16)
        return err(MLEM_ERR_FORMAT, "Input file '%s' has an impossible element count", path);
    const uint64_t need = (uint64_t)kHeaderBytes + h->scan_config_bytes + 8ull * h->n_rows + 8ull * h->nnz;
    if (size < need)
        return err(MLEM_ERR_FORMAT, "Input file '%s' is too short: %llu B instead of at least %llu B",
                   path, (unsigned long long)size, (unsigned long long)need);
    if (h->scan_config_bytes < kMinScanConfig)
        return err(MLEM_ERR_FORMAT, "Cannot find scanner geometry configuration");
    // scanner geometry block, csr4matrix.cpp:100-138
    const unsigned char* p = head + kHeaderBytes;
    const unsigned char* end = head + hl;
    auto need_bytes = [&](size_t n) { return p + n <= end; };
    if (!need_bytes(4)) return err(MLEM_ERR_FORMAT, "Error reading scanner geometry configuration");
    const uint32_t n_layers = rd<uint32_t>(p); p += 4;
    if ((uint64_t)n_layers * 20 > (uint64_t)(end - p))
        return err(MLEM_ERR_FORMAT, "Error reading scanner geometry configuration");
    p += 20ull * n_layers;
    if (!need_bytes(8)) return err(MLEM_ERR_FORMAT, "Error reading scanner geometry configuration");
    const uint32_t n_blocks = rd<uint32_t>(p); p += 4;
    const uint32_t blocksize = rd<uint32_t>(p); p += 4;
    const uint64_t block_gaps = blocksize ? blocksize - 1ull : 0;
    if (block_gaps * 4 + 4 > (uint64_t)(end - p))
        return err(MLEM_ERR_FORMAT, "Error reading scanner geometry configuration");
    p += 4 * block_gaps;
    const uint32_t n_rings = rd<uint32_t>(p); p += 4;
    const uint64_t ring_gaps = n_rings ? n_rings - 1ull : 0;
    if (ring_gaps * 4 + 24 > (uint64_t)(end - p))
        return err(MLEM_ERR_FORMAT, "Error reading scanner geometry configuration");
    p += 4 * ring_gaps;
    for (int i = 0; i < 3; ++i) { h->voxel_size[i] = rd<float>(p); p += 4; }
    for (int i = 0; i < 3; ++i) { h->grid[i] = rd<uint32_t>(p); p += 4; }
    if ((uint64_t)(p - (head + kHeaderBytes)) != h->scan_config_bytes)
        return err(MLEM_ERR_FORMAT, "Error reading scanner geometry configuration");
    h->data_offset = kHeaderBytes + h->scan_config_bytes;
    h->n_layers = n_layers;
    h->n_blocks = n_blocks;
    h->block_size = blocksize;
    h->n_rings = n_rings;
    return MLEM_OK;
}

const char* checkpoint_path(std::string& buf, const char* dir, const char* name) {
    buf = (dir && *dir) ? std::string(dir) + "/" + name : std::string(name);
    return buf.c_str();
}

}  // namespace
}  // namespace mlem

using namespace mlem;

extern "C" {

int mlem_csr4_read_header(const char* path, mlem_csr4_header* out) {
    if (!path || !out) return err(MLEM_ERR_INVALID, "null argument");
    Fd f;
    f.fd = ::open(path, O_RDONLY);
    if (f.fd < 0) return err(MLEM_ERR_IO, "Cannot open file %s", path);
    return parse_header(path, f.fd, out);
}

int mlem_csr4_read(const char* path, uint64_t* row_end, void* elems) {
    if (!path) return err(MLEM_ERR_INVALID, "null path");
    Fd f;
    f.fd = ::open(path, O_RDONLY);
    if (f.fd < 0) return err(MLEM_ERR_IO, "Cannot open file %s", path);
    mlem_csr4_header h;
    int s = parse_header(path, f.fd, &h);
    if (s != MLEM_OK) return s;
    if (row_end && h.n_rows &&
        !read_full(f.fd, row_end, 8ull * h.n_rows, (off_t)h.data_offset))
        return err(MLEM_ERR_IO, "Cannot read row indexes %s", path);
    if (elems && h.nnz &&
        !read_full(f.fd, elems, 8ull * h.nnz, (off_t)(h.data_offset + 8ull * h.n_rows)))
        return err(MLEM_ERR_IO, "Cannot read matrix elements %s", path);
    return MLEM_OK;
}

int mlem_csr4_write(const char* path, const uint64_t* row_end, const void* elems, uint32_t n_rows,
                    uint32_t n_cols, const uint32_t grid[3]) {
    if (!path || (n_rows && !row_end)) return err(MLEM_ERR_INVALID, "null argument");
    const uint64_t nnz = n_rows ? row_end[n_rows - 1] : 0;
    if (nnz && !elems) return err(MLEM_ERR_INVALID, "null elements");
    unsigned char head[kHeaderBytes + kMinScanConfig];
    std::memset(head, 0, sizeof(head));
    std::memcpy(head, "PCSR", 4);
    head[4] = 4;
    std::memcpy(head + 8, &n_rows, 4);
    std::memcpy(head + 12, &n_cols, 4);
    std::memcpy(head + 16, &nnz, 8);
    const uint32_t scb = kMinScanConfig;
    std::memcpy(head + 24, &scb, 4);
    unsigned char* p = head + kHeaderBytes;
    const uint32_t one = 1;
    const float layer[5] = {1.0f, 1.0f, 1.0f, 1.0f, 0.0f};
    const float vox[3] = {1.0f, 1.0f, 1.0f};
    const uint32_t g[3] = {grid ? grid[0] : 0u, grid ? grid[1] : 0u, grid ? grid[2] : 0u};
    std::memcpy(p, &one, 4); p += 4;            // nLayers
    std::memcpy(p, layer, 20); p += 20;         // w, h, d, r, mu
    std::memcpy(p, &one, 4); p += 4;            // nBlocks
    std::memcpy(p, &one, 4); p += 4;            // blocksize (no gaps)
    std::memcpy(p, &one, 4); p += 4;            // nRings (no gaps)
    std::memcpy(p, vox, 12); p += 12;           // voxel size
    std::memcpy(p, g, 12); p += 12;             // grid
    Fd f;
    f.fd = ::open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (f.fd < 0) return err(MLEM_ERR_IO, "Cannot open file %s; reason: %s", path, strerror(errno));
    if (!write_full(f.fd, head, sizeof(head)) ||
        (n_rows && !write_full(f.fd, row_end, 8ull * n_rows)) ||
        (nnz && !write_full(f.fd, elems, 8ull * nnz)))
        return err(MLEM_ERR_IO, "Cannot write file %s; reason: %s", path, strerror(errno));
    return MLEM_OK;
}

int mlem_vector_read(const char* path, uint32_t elem_size, void* buf, uint64_t capacity,
                     uint64_t* count) {
    if (!path || elem_size == 0) return err(MLEM_ERR_INVALID, "bad argument");
    Fd f;
    f.fd = ::open(path, O_RDONLY);
    if (f.fd < 0) return err(MLEM_ERR_IO, "Cannot open file %s", path);
    struct stat st;
    if (::fstat(f.fd, &st) != 0) return err(MLEM_ERR_IO, "Cannot open file %s", path);
    const uint64_t bytes = (uint64_t)st.st_size;
    if (bytes % elem_size)  // vector.hpp:43-44
        return err(MLEM_ERR_FORMAT, "Cannot open file %s (size %llu is not a multiple of %u)", path,
                   (unsigned long long)bytes, elem_size);
    const uint64_t n = bytes / elem_size;
    if (count) *count = n;
    if (!buf) return MLEM_OK;
    if (n > capacity)
        return err(MLEM_ERR_INVALID, "file %s holds %llu elements, buffer %llu", path,
                   (unsigned long long)n, (unsigned long long)capacity);
    if (n && !read_full(f.fd, buf, bytes, 0)) return err(MLEM_ERR_IO, "Cannot read file %s", path);
    return MLEM_OK;
}

int mlem_vector_write(const char* path, const void* buf, uint32_t elem_size, uint64_t count,
                      int sync) {
    if (!path || (count && !buf)) return err(MLEM_ERR_INVALID, "null argument");
    Fd f;
    f.fd = ::open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (f.fd < 0)
        return err(MLEM_ERR_IO, "Cannot open file %s; reason: %s", path, strerror(errno));
    if (count && !write_full(f.fd, buf, (size_t)count * elem_size))
        return err(MLEM_ERR_IO, "Cannot write file %s; reason: %s", path, strerror(errno));
    if (sync && ::fsync(f.fd) != 0)  // vector.hpp:111-112
        return err(MLEM_ERR_IO, "Cannot sync file %s; reason: %s", path, strerror(errno));
    return MLEM_OK;
}

int mlem_checkpoint_write(const char* dir, const float* image, uint32_t n_cols, int32_t next_iter) {
    std::string a, b;
    // image first, then the iteration number, each fsync'd (mpicsr4mlem.cpp:107-121)
    int s = mlem_vector_write(checkpoint_path(a, dir, "img.chkpt"), image, 4, n_cols, 1);
    if (s != MLEM_OK) return s;
    return mlem_vector_write(checkpoint_path(b, dir, "iter.chkpt"), &next_iter, 4, 1, 1);
}

int mlem_checkpoint_read(const char* dir, float* image, uint32_t n_cols, int32_t* next_iter) {
    std::string a, b;
    const char* img = checkpoint_path(a, dir, "img.chkpt");
    const char* itr = checkpoint_path(b, dir, "iter.chkpt");
    struct stat st;
    const bool has_img = ::stat(img, &st) == 0, has_itr = ::stat(itr, &st) == 0;
    if (!(has_img && has_itr)) {
        // mpicsr4mlem.cpp:545-550: an incomplete checkpoint is ignored
        return set_error(nullptr, MLEM_NO_CHECKPOINT, "%s",
                         (has_img || has_itr) ? "omitted incomplete checkpoint" : "no checkpoint");
    }
    uint64_t n = 0;
    int s = mlem_vector_read(img, 4, nullptr, 0, &n);
    if (s != MLEM_OK) return s;
    if (n != n_cols)  // vector.hpp:131-134
        return err(MLEM_ERR_FORMAT, "Mismatch element number %s (%llu, expected %u)", img,
                   (unsigned long long)n, n_cols);
    s = mlem_vector_read(img, 4, image, n_cols, &n);
    if (s != MLEM_OK) return s;
    int32_t it = 0;
    uint64_t m = 0;
    s = mlem_vector_read(itr, 4, nullptr, 0, &m);
    if (s != MLEM_OK) return s;
    if (m < 1) return err(MLEM_ERR_FORMAT, "Cannot read iteration from %s", itr);
    Fd f;
    f.fd = ::open(itr, O_RDONLY);
    if (f.fd < 0 || !read_full(f.fd, &it, 4, 0)) return err(MLEM_ERR_IO, "Cannot open file %s", itr);
    if (it < 0) return err(MLEM_ERR_FORMAT, "negative iteration %d in %s", it, itr);
    *next_iter = it;
    return MLEM_OK;
}

int mlem_checkpoint_remove(const char* dir) {
    std::string a, b;
    ::remove(checkpoint_path(a, dir, "img.chkpt"));
    ::remove(checkpoint_path(b, dir, "iter.chkpt"));
    return MLEM_OK;
}

int mlem_partition_rows(const uint64_t* row_end, uint32_t n_rows, int n_ranks, uint32_t* starts,
                        uint32_t* ends) {
    if (n_ranks < 1 || !starts || !ends || (n_rows && !row_end))
        return err(MLEM_ERR_INVALID, "bad argument");
    // mpicsr4mlem.cpp:206-224, including its float comparison of the running sum
    const uint64_t Z = n_rows ? row_end[n_rows - 1] : 0;
    const float avg = (float)Z / (float)n_ranks;
    for (int i = 0; i < n_ranks; ++i) { starts[i] = 0; ends[i] = 0; }
    int idx = 0;
    uint64_t sum = 0, prev = 0;
    for (uint32_t r = 0; r < n_rows; ++r) {
        sum += row_end[r] - prev;
        prev = row_end[r];
        if ((float)sum > avg * (float)(idx + 1) && idx + 1 < n_ranks) {
            ends[idx] = r + 1;
            idx += 1;
            starts[idx] = r + 1;
        }
    }
    for (int i = idx + 1; i < n_ranks; ++i) starts[i] = n_rows;
    for (int i = idx; i < n_ranks; ++i) ends[i] = n_rows;
    return MLEM_OK;
}

int mlem_create_from_file(mlem_ctx** out, const char* path, uint32_t flags, int device) {
    if (!out || !path) return err(MLEM_ERR_INVALID, "null argument");
    *out = nullptr;
    Fd f;
    f.fd = ::open(path, O_RDONLY);
    if (f.fd < 0) return err(MLEM_ERR_IO, "Cannot open file %s", path);
    mlem_csr4_header h;
    int s = parse_header(path, f.fd, &h);
    if (s != MLEM_OK) return s;
    // Map the whole file read-only (csr4matrix.cpp:209 maps the element region
    // the same way) and upload straight from the mapping.
    void* map = nullptr;
    if (h.file_size) {
        map = ::mmap(nullptr, h.file_size, PROT_READ, MAP_PRIVATE, f.fd, 0);
        if (map == MAP_FAILED) return err(MLEM_ERR_IO, "Cannot map file %s", path);
    }
    const unsigned char* base = static_cast<const unsigned char*>(map);
    const uint64_t* row_end = reinterpret_cast<const uint64_t*>(base + h.data_offset);
    const void* elems = base + h.data_offset + 8ull * h.n_rows;
    std::vector<uint64_t> aligned;
    if (h.data_offset % 8) {  // non-standard scanner block size: copy to align the offsets
        aligned.resize(h.n_rows);
        std::memcpy(aligned.data(), base + h.data_offset, 8ull * h.n_rows);
        row_end = aligned.data();
    }
    const uint32_t sym_flags = MLEM_FLAG_EXPAND_SYMMETRY | MLEM_FLAG_MIRROR_KERNELS;
    if ((flags & MLEM_FLAG_EXPAND_SYMMETRY) && (flags & MLEM_FLAG_MIRROR_KERNELS)) {
        s = err(MLEM_ERR_INVALID,
                "MLEM_FLAG_EXPAND_SYMMETRY and MLEM_FLAG_MIRROR_KERNELS exclude each other");
    } else if ((flags & sym_flags) && (h.flags & 7u)) {
        // the elements the symmetries omitted: regenerated (expand) or applied
        // in the kernels (the reference's MLEM would use the stored ones only)
        mlem_symmetry sym{h.flags & 7u, h.n_layers, h.n_blocks, h.block_size, h.n_rings,
                          {h.grid[0], h.grid[1], h.grid[2]}};
        s = mlem_create_symmetric(out, row_end, elems, h.n_rows, h.n_cols, h.nnz, &sym,
                                  flags & ~MLEM_FLAG_EXPAND_SYMMETRY, device);
    } else {
        s = mlem_create_grid(out, row_end, elems, h.n_rows, h.n_cols, h.nnz, h.grid,
                             flags & ~sym_flags, device);
    }
    if (map) ::munmap(map, h.file_size);
    return s;
}

}  // extern "C"
