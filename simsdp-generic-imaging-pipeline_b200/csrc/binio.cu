// Binary on-disk formats for the imaging inputs, and their loading straight
// into device memory.
//
// The reference reads its inputs as text (top.c:139-222 visibilities,
// :224-380 kernel tables, :453-510 the PSF), which dominates its end-to-end
// time.  These files hold the same arrays as raw little-endian floats behind
// a 64-byte header, so a load is one sequential read:
//
//   header  "SDPBIN1" + kind (1 visibilities, 2 kernel set, 3 image),
//           count, aux, payload sections (offset, bytes) x 2
//   kind 1: uvw float32[n][3] (metres = wavelengths, as the reference's CSV
//           carries them; aux bit 0 set when they are already snapped by
//           correct_to_finegrid) | vis float32[n][2]
//   kind 2: supports int32[planes][2] (half support, sample offset, as
//           kernel_host_set_up builds them, top.c:256-261) | samples
//           float32[total][2]; count = total samples, aux = planes
//   kind 3: float32[rows][cols]; count = rows, aux = cols
//
// Sections start on 4096-byte boundaries.  Device loads read the file in
// chunks into a ring of pinned host buffers with several threads (pread),
// and each filled chunk goes to the device with cudaMemcpyAsync on the
// caller's stream while the next chunk is read; a chunk's buffer is reused
// only after the event recorded behind its copy has completed.  The call
// returns when every copy has been issued and the ring has drained.
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "common.cuh"

namespace sdp {
namespace {

constexpr char kMagic[8] = {'S', 'D', 'P', 'B', 'I', 'N', '1', '\0'};
constexpr uint64_t kAlign = 4096;
constexpr size_t kChunk = 32u << 20;  // bytes per staging buffer
constexpr int kRing = 4;              // staging buffers in flight

struct Header {
    char magic[8];
    uint32_t kind;
    uint32_t version;
    uint64_t count;
    uint64_t aux;
    uint64_t off[2];
    uint64_t bytes[2];
};
static_assert(sizeof(Header) == 64, "header is 64 bytes");

uint64_t align_up(uint64_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

struct Fd {
    int fd = -1;
    ~Fd()
    {
        if (fd >= 0) close(fd);
    }
};

int write_all(int fd, const void *p, size_t n, uint64_t off, const char *path)
{
    const char *c = static_cast<const char *>(p);
    while (n > 0) {
        const ssize_t w = pwrite(fd, c, std::min<size_t>(n, 1u << 30), (off_t)off);
        if (w < 0) {
            if (errno == EINTR) continue;
            return set_error(SDP_ERR_IO, "writing %s: %s", path, std::strerror(errno));
        }
        c += w;
        off += (uint64_t)w;
        n -= (size_t)w;
    }
    return SDP_OK;
}

int read_all(int fd, void *p, size_t n, uint64_t off, const char *path)
{
    char *c = static_cast<char *>(p);
    while (n > 0) {
        const ssize_t r = pread(fd, c, std::min<size_t>(n, 1u << 30), (off_t)off);
        if (r < 0) {
            if (errno == EINTR) continue;
            return set_error(SDP_ERR_IO, "reading %s: %s", path, std::strerror(errno));
        }
        if (r == 0) return set_error(SDP_ERR_IO, "%s: file ends early", path);
        c += r;
        off += (uint64_t)r;
        n -= (size_t)r;
    }
    return SDP_OK;
}

// Reads [off, off + n) with up to `threads` concurrent preads.
int read_parallel(int fd, void *p, size_t n, uint64_t off, const char *path, int threads)
{
    if (threads <= 1 || n < (4u << 20)) return read_all(fd, p, n, off, path);
    const size_t part = (n + threads - 1) / threads;
    std::vector<int> st((size_t)threads, SDP_OK);
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) {
        const size_t b = (size_t)t * part;
        if (b >= n) break;
        const size_t len = std::min(part, n - b);
        pool.emplace_back([&, t, b, len] { st[(size_t)t] = read_all(fd, static_cast<char *>(p) + b, len, off + b, path); });
    }
    for (auto &th : pool) th.join();
    for (int s : st)
        if (s != SDP_OK) return set_error(SDP_ERR_IO, "reading %s failed", path);
    return SDP_OK;
}

int open_checked(const char *path, int kind, Header &h, Fd &f)
{
    if (!path) return set_error(SDP_ERR_INVALID, "file name is NULL");
    f.fd = open(path, O_RDONLY);
    if (f.fd < 0) return set_error(SDP_ERR_IO, "unable to open %s: %s", path, std::strerror(errno));
    SDP_TRY(read_all(f.fd, &h, sizeof(h), 0, path));
    if (std::memcmp(h.magic, kMagic, 8) != 0 || h.version != 1)
        return set_error(SDP_ERR_DATA, "%s is not an sdp binary file (version 1)", path);
    if (kind && (int)h.kind != kind) return set_error(SDP_ERR_DATA, "%s holds kind %u, not %d", path, h.kind, kind);
    struct stat s;
    if (fstat(f.fd, &s) != 0) return set_error(SDP_ERR_IO, "unable to stat %s", path);
    for (int k = 0; k < 2; ++k)
        if (h.bytes[k] && h.off[k] + h.bytes[k] > (uint64_t)s.st_size)
            return set_error(SDP_ERR_DATA, "%s: section %d runs past the end of the file", path, k);
    return SDP_OK;
}

int write_file(const char *path, uint32_t kind, uint64_t count, uint64_t aux, const void *a, uint64_t na,
               const void *b, uint64_t nb)
{
    if (!path) return set_error(SDP_ERR_INVALID, "file name is NULL");
    Header h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, kMagic, 8);
    h.kind = kind;
    h.version = 1;
    h.count = count;
    h.aux = aux;
    h.off[0] = kAlign;
    h.bytes[0] = na;
    h.off[1] = align_up(kAlign + na);
    h.bytes[1] = nb;
    Fd f;
    f.fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (f.fd < 0) return set_error(SDP_ERR_IO, "unable to create %s: %s", path, std::strerror(errno));
    SDP_TRY(write_all(f.fd, &h, sizeof(h), 0, path));
    if (na) SDP_TRY(write_all(f.fd, a, (size_t)na, h.off[0], path));
    if (nb) SDP_TRY(write_all(f.fd, b, (size_t)nb, h.off[1], path));
    // the file ends at the last section (no trailing padding)
    if (ftruncate(f.fd, (off_t)(nb ? h.off[1] + nb : h.off[0] + na)) != 0)
        return set_error(SDP_ERR_IO, "sizing %s: %s", path, std::strerror(errno));
    return SDP_OK;
}

int host_threads()
{
    const unsigned n = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(n, 8u));
}

// The staging ring of one thread: pinned buffers and their events.
struct Ring {
    void *buf[kRing] = {};
    cudaEvent_t ev[kRing] = {};
    int dev = -1;
    ~Ring()
    {
        for (int k = 0; k < kRing; ++k) {
            if (buf[k]) cudaFreeHost(buf[k]);
            if (ev[k]) cudaEventDestroy(ev[k]);
        }
    }
};
thread_local Ring t_ring;

int ring_ready(Ring &r)
{
    int dev = 0;
    SDP_CUDA_TRY(cudaGetDevice(&dev));
    if (r.buf[0] && r.dev == dev) return SDP_OK;
    for (int k = 0; k < kRing; ++k) {
        if (!r.buf[k]) SDP_CUDA_TRY(cudaHostAlloc(&r.buf[k], kChunk, cudaHostAllocDefault));
        if (r.ev[k]) cudaEventDestroy(r.ev[k]);
        r.ev[k] = nullptr;
        SDP_CUDA_TRY(cudaEventCreateWithFlags(&r.ev[k], cudaEventDisableTiming));
    }
    r.dev = dev;
    return SDP_OK;
}

// File section [off, off + n) -> device dst, through the staging ring.
int stage_to_device(int fd, uint64_t off, size_t n, void *dst, const char *path, cudaStream_t st)
{
    Ring &r = t_ring;
    SDP_TRY(ring_ready(r));
    const int threads = host_threads();
    bool used[kRing] = {};
    size_t done = 0;
    int k = 0;
    while (done < n) {
        const size_t len = std::min(kChunk, n - done);
        if (used[k]) SDP_CUDA_TRY(cudaEventSynchronize(r.ev[k]));  // its previous copy has finished
        SDP_TRY(read_parallel(fd, r.buf[k], len, off + done, path, threads));
        SDP_CUDA_TRY(cudaMemcpyAsync(static_cast<char *>(dst) + done, r.buf[k], len, cudaMemcpyHostToDevice, st));
        SDP_CUDA_TRY(cudaEventRecord(r.ev[k], st));
        used[k] = true;
        done += len;
        k = (k + 1) % kRing;
    }
    for (int j = 0; j < kRing; ++j)
        if (used[j]) SDP_CUDA_TRY(cudaEventSynchronize(r.ev[j]));
    return SDP_OK;
}

}  // namespace
}  // namespace sdp

using namespace sdp;

SDP_EXPORT int sdp_bin_info(const char *path, int *kind, long long *count, long long *aux)
{
    SDP_CHECK_ARG(kind && count && aux, "NULL argument");
    Header h;
    Fd f;
    SDP_TRY(open_checked(path, 0, h, f));
    *kind = (int)h.kind;
    *count = (long long)h.count;
    *aux = (long long)h.aux;
    return SDP_OK;
}

SDP_EXPORT int sdp_bin_write_vis(const char *path, long long num_vis, const sdp_float3 *uvw, const sdp_float2 *vis,
                                 int snapped)
{
    SDP_CHECK_ARG(num_vis >= 0 && (num_vis == 0 || (uvw && vis)), "bad visibility arrays");
    return write_file(path, 1, (uint64_t)num_vis, snapped ? 1u : 0u, uvw, (uint64_t)num_vis * 12, vis,
                      (uint64_t)num_vis * 8);
}

SDP_EXPORT int sdp_bin_write_kernels(const char *path, int num_planes, long long total_samples,
                                     const sdp_int2 *supports, const sdp_float2 *samples)
{
    SDP_CHECK_ARG(num_planes >= 1 && total_samples >= 0 && supports && (samples || total_samples == 0),
                  "bad kernel arrays");
    return write_file(path, 2, (uint64_t)total_samples, (uint64_t)num_planes, supports, (uint64_t)num_planes * 8,
                      samples, (uint64_t)total_samples * 8);
}

SDP_EXPORT int sdp_bin_write_image(const char *path, int rows, int cols, const float *image)
{
    SDP_CHECK_ARG(rows >= 1 && cols >= 1 && image, "bad image");
    return write_file(path, 3, (uint64_t)rows, (uint64_t)cols, image, (uint64_t)rows * cols * 4, nullptr, 0);
}

// Host reads (for callers that stage themselves, and for tests).
SDP_EXPORT int sdp_bin_read_vis_host(const char *path, long long max_vis, sdp_float3 *uvw, sdp_float2 *vis,
                                     long long *num_vis, int *snapped)
{
    SDP_CHECK_ARG(uvw && vis && num_vis, "NULL argument");
    Header h;
    Fd f;
    SDP_TRY(open_checked(path, 1, h, f));
    if ((long long)h.count > max_vis)
        return set_error(SDP_ERR_RANGE, "%s holds %llu visibilities, buffers hold %lld", path,
                         (unsigned long long)h.count, max_vis);
    if (h.bytes[0] != h.count * 12 || h.bytes[1] != h.count * 8)
        return set_error(SDP_ERR_DATA, "%s: section sizes do not match the count", path);
    SDP_TRY(read_parallel(f.fd, uvw, (size_t)h.bytes[0], h.off[0], path, host_threads()));
    SDP_TRY(read_parallel(f.fd, vis, (size_t)h.bytes[1], h.off[1], path, host_threads()));
    *num_vis = (long long)h.count;
    if (snapped) *snapped = (int)(h.aux & 1);
    return SDP_OK;
}

// Device loads: the arrays land in device memory through pinned staging.
SDP_EXPORT int sdp_bin_load_vis(const char *path, long long max_vis, sdp_float3 *uvw_dev, sdp_float2 *vis_dev,
                                long long *num_vis, int *snapped, void *stream)
{
    SDP_CHECK_ARG(uvw_dev && vis_dev && num_vis, "NULL argument");
    Header h;
    Fd f;
    SDP_TRY(open_checked(path, 1, h, f));
    if ((long long)h.count > max_vis)
        return set_error(SDP_ERR_RANGE, "%s holds %llu visibilities, buffers hold %lld", path,
                         (unsigned long long)h.count, max_vis);
    if (h.bytes[0] != h.count * 12 || h.bytes[1] != h.count * 8)
        return set_error(SDP_ERR_DATA, "%s: section sizes do not match the count", path);
    cudaStream_t st = as_stream(stream);
    SDP_TRY(stage_to_device(f.fd, h.off[0], (size_t)h.bytes[0], uvw_dev, path, st));
    SDP_TRY(stage_to_device(f.fd, h.off[1], (size_t)h.bytes[1], vis_dev, path, st));
    *num_vis = (long long)h.count;
    if (snapped) *snapped = (int)(h.aux & 1);
    return SDP_OK;
}

SDP_EXPORT int sdp_bin_load_kernels(const char *path, int max_planes, long long max_samples, sdp_int2 *supports_dev,
                                    sdp_float2 *samples_dev, int *num_planes, long long *total_samples, void *stream)
{
    SDP_CHECK_ARG(supports_dev && samples_dev && num_planes && total_samples, "NULL argument");
    Header h;
    Fd f;
    SDP_TRY(open_checked(path, 2, h, f));
    if ((long long)h.aux > max_planes || (long long)h.count > max_samples)
        return set_error(SDP_ERR_RANGE, "%s: %llu planes / %llu samples exceed the buffers", path,
                         (unsigned long long)h.aux, (unsigned long long)h.count);
    if (h.bytes[0] != h.aux * 8 || h.bytes[1] != h.count * 8)
        return set_error(SDP_ERR_DATA, "%s: section sizes do not match the counts", path);
    cudaStream_t st = as_stream(stream);
    SDP_TRY(stage_to_device(f.fd, h.off[0], (size_t)h.bytes[0], supports_dev, path, st));
    SDP_TRY(stage_to_device(f.fd, h.off[1], (size_t)h.bytes[1], samples_dev, path, st));
    *num_planes = (int)h.aux;
    *total_samples = (long long)h.count;
    return SDP_OK;
}

SDP_EXPORT int sdp_bin_load_image(const char *path, int max_rows, int max_cols, float *image_dev, int *rows,
                                  int *cols, void *stream)
{
    SDP_CHECK_ARG(image_dev && rows && cols, "NULL argument");
    Header h;
    Fd f;
    SDP_TRY(open_checked(path, 3, h, f));
    if ((long long)h.count > max_rows || (long long)h.aux > max_cols)
        return set_error(SDP_ERR_RANGE, "%s: %llu x %llu image exceeds the buffer", path, (unsigned long long)h.count,
                         (unsigned long long)h.aux);
    if (h.bytes[0] != h.count * h.aux * 4) return set_error(SDP_ERR_DATA, "%s: section size does not match", path);
    SDP_TRY(stage_to_device(f.fd, h.off[0], (size_t)h.bytes[0], image_dev, path, as_stream(stream)));
    *rows = (int)h.count;
    *cols = (int)h.aux;
    return SDP_OK;
}
