// File-reading set-up actors (param_code/code_fft_1core/src/top.c):
//   visibility_host_set_up         top.c:139-222
//   kernel_host_set_up             top.c:224-300
//   degridding_kernel_host_set_up  top.c:303-380
//   psf_host_set_up                top.c:453-510
//
// The reference reads its text inputs one fscanf("%lf") at a time, which
// dominates its end-to-end time (a 3.9 M-visibility file is ~280 MB of
// text).  Here the whole file is mapped and split into whitespace separated
// tokens by several host threads (a counting pass, then each thread converts
// its range into its slice of the output); each token is converted with
// std::from_chars (correctly rounded, as glibc's strtod that fscanf uses),
// falling back to strtod for spellings from_chars does not take.  After
// parsing, the reference's per-record arithmetic runs unchanged (double
// products rounded to float where it assigns, fabsf for ABS in the float
// build), including its behaviour on short files: fscanf leaves its target
// variables unchanged once the input ends, and the loops then keep
// transforming the stale values, which is replayed exactly.  A token that is
// not a number ends the input, as it stops fscanf for good.
//
// Host code only: these actors touch no GPU.
#include <cerrno>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"

namespace {

using sdp::set_error;

bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }

// A read-only view of a whole file (mapped, so nothing is copied).
struct FileView {
    const char *data = nullptr;
    size_t size = 0;
    int fd = -1;
    void *map = nullptr;
    ~FileView()
    {
        if (map) munmap(map, size);
        if (fd >= 0) close(fd);
    }
};

int read_file(const char *path, FileView &f)
{
    if (!path) return set_error(SDP_ERR_INVALID, "file name is NULL");
    f.fd = open(path, O_RDONLY);
    if (f.fd < 0) return set_error(SDP_ERR_IO, "unable to open %s: %s", path, std::strerror(errno));
    struct stat st;
    if (fstat(f.fd, &st) != 0) return set_error(SDP_ERR_IO, "unable to stat %s: %s", path, std::strerror(errno));
    f.size = (size_t)st.st_size;
    if (f.size == 0) return SDP_OK;
    f.map = mmap(nullptr, f.size, PROT_READ, MAP_PRIVATE | MAP_POPULATE, f.fd, 0);
    if (f.map == MAP_FAILED) {
        f.map = nullptr;
        return set_error(SDP_ERR_IO, "unable to map %s: %s", path, std::strerror(errno));
    }
    f.data = static_cast<const char *>(f.map);
    return SDP_OK;
}

// One %lf conversion of the token [b, e).  Returns 0: not a number (fscanf
// would fail here); 1: the whole token converted; 2: a leading part
// converted (the next conversion would fail on the rest).
int parse_double(const char *b, const char *e, double *out)
{
    const char *s = b;
    if (s < e && *s == '+') ++s;
    if (s < e && !(s + 1 < e && s[0] == '0' && (s[1] == 'x' || s[1] == 'X'))) {
        auto r = std::from_chars(s, e, *out, std::chars_format::general);
        if (r.ec == std::errc() && r.ptr == e) return 1;
        if (r.ec == std::errc::result_out_of_range) {
            // strtod gives +-HUGE_VAL / denormal results; take its value below
        }
    }
    char tmp[128];
    const size_t len = std::min<size_t>((size_t)(e - b), sizeof(tmp) - 1);
    std::memcpy(tmp, b, len);
    tmp[len] = '\0';
    char *end = nullptr;
    *out = std::strtod(tmp, &end);
    if (end == tmp) return 0;
    return (size_t)(end - tmp) == (size_t)(e - b) ? 1 : 2;
}

// First token start at or after b (a token that starts before b belongs to
// the previous range; `from`, where the input resumes, is a start itself,
// as after fscanf's "%d" took the leading digits of a token).
size_t first_token(const char *buf, size_t b, size_t size, size_t from)
{
    size_t i = b;
    if (i > from && i < size && !is_space(buf[i - 1]))
        while (i < size && !is_space(buf[i])) ++i;
    return i;
}

size_t count_tokens(const char *buf, size_t b, size_t e, size_t size, size_t from)
{
    size_t n = 0;
    size_t i = first_token(buf, b, size, from);
    while (true) {
        while (i < size && is_space(buf[i])) ++i;
        if (i >= size || i >= e) break;
        ++n;
        while (i < size && !is_space(buf[i])) ++i;
    }
    return n;
}

// Converts the tokens starting in [b, e) into out[0..]; returns how many
// converted before a token that ends the input (*stop set then).
size_t parse_range(const char *buf, size_t b, size_t e, size_t size, size_t from, double *out, bool *stop)
{
    size_t n = 0;
    size_t i = first_token(buf, b, size, from);
    *stop = false;
    while (true) {
        while (i < size && is_space(buf[i])) ++i;
        if (i >= size || i >= e) break;
        size_t j = i;
        while (j < size && !is_space(buf[j])) ++j;
        double x = 0.0;
        const int k = parse_double(buf + i, buf + j, &x);
        if (k == 0) {
            *stop = true;
            break;
        }
        out[n++] = x;
        if (k == 2) {
            *stop = true;
            break;
        }
        i = j;
    }
    return n;
}

// All numbers of the file from byte `from`, in order, up to the first token
// that is not (wholly) a number.  Threads count their ranges' tokens, then
// convert straight into their slice of the output.
void parse_all(const FileView &f, size_t from, std::vector<double> &out)
{
    const size_t size = f.size;
    const char *buf = f.data;
    from = std::min(from, size);
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (size - from < (1u << 20)) nt = 1;
    const size_t span = (size - from + nt - 1) / nt;
    std::vector<size_t> cnt(nt), got(nt);
    std::vector<char> stop(nt, 0);
    auto run = [&](auto &&fn) {
        std::vector<std::thread> th;
        for (unsigned t = 1; t < nt; ++t) th.emplace_back(fn, t);
        fn(0u);
        for (auto &x : th) x.join();
    };
    run([&](unsigned t) {
        cnt[t] = count_tokens(buf, std::min(size, from + t * span), std::min(size, from + (t + 1) * span), size, from);
    });
    std::vector<size_t> off(nt + 1, 0);
    for (unsigned t = 0; t < nt; ++t) off[t + 1] = off[t] + cnt[t];
    out.resize(off[nt]);
    run([&](unsigned t) {
        bool st = false;
        got[t] = parse_range(buf, std::min(size, from + t * span), std::min(size, from + (t + 1) * span), size, from,
                             out.data() + off[t], &st);
        stop[t] = st;
    });
    // the input ends at the first range that stopped early
    for (unsigned t = 0; t < nt; ++t)
        if (stop[t] || got[t] < cnt[t]) {
            out.resize(off[t] + got[t]);
            break;
        }
}

// The first token as fscanf("%d") reads it; returns the byte after it.
size_t parse_leading_int(const FileView &f, int *value, bool *ok)
{
    size_t i = 0;
    while (i < f.size && is_space(f.data[i])) ++i;
    size_t j = i;
    while (j < f.size && !is_space(f.data[j]) && j - i < 63) ++j;
    char tmp[64];
    std::memcpy(tmp, f.data + i, j - i);
    tmp[j - i] = '\0';
    char *end = nullptr;
    const long v = std::strtol(tmp, &end, 10);
    *ok = end != tmp;
    if (*ok) *value = (int)v;
    return i + (size_t)(end - tmp);
}

// "%d\n" per plane into supports[p].x, offsets into .y (top.c:246-251).
int read_supports(const char *path, int nk, int os, sdp_int2 *sup)
{
    FileView f;
    SDP_TRY(read_file(path, f));
    const std::string buf(f.data ? f.data : "", f.size);  // small file: a terminated copy for strtol
    const char *s = buf.c_str();
    int total = 0;
    for (int p = 0; p < nk; ++p) {
        char *end = nullptr;
        const long v = std::strtol(s, &end, 10);
        if (end != s) {
            sup[p].x = (int)v;
            s = end;
        }  // a failed conversion leaves .x as it was
        sup[p].y = total;
        total += (int)std::pow((double)((sup[p].x + 1) * os), 2.0);
    }
    return SDP_OK;
}

int load_kernels(const char *sup_file, const char *re_file, const char *im_file, int nk, int os, sdp_int2 *sup,
                 sdp_float2 *kernels)
{
    SDP_TRY(read_supports(sup_file, nk, os, sup));
    FileView rb, ib;
    SDP_TRY(read_file(re_file, rb));
    SDP_TRY(read_file(im_file, ib));
    std::vector<double> re, im;
    parse_all(rb, 0, re);
    parse_all(ib, 0, im);
    size_t k = 0;
    for (int p = 0; p < nk; ++p) {
        const int ns = (int)std::pow((double)((sup[p].x + 1) * os), 2.0);
        for (int j = 0; j < ns; ++j, ++k) {
            // real and imag start at 0.0 for every sample (top.c:283-284)
            kernels[k].x = (float)(k < re.size() ? re[k] : 0.0);
            kernels[k].y = (float)(k < im.size() ? im[k] : 0.0);
        }
    }
    return SDP_OK;
}

int load_visibilities(int n, const sdp_config *cfg, sdp_float3 *uvw, sdp_float2 *vis)
{
    SDP_CHECK_ARG(cfg && (n == 0 || (uvw && vis)), "bad argument");
    FileView buf;
    SDP_TRY(read_file(cfg->visibility_source_file, buf));
    int count = 0;
    bool ok = false;
    const size_t after = parse_leading_int(buf, &count, &ok);
    std::vector<double> t;
    if (ok) parse_all(buf, after, t);  // a failed %d stops every later conversion too
    const double m2w = cfg->frequency_hz / 299792458.0;  // SPEED_OF_LIGHT
    const bool ra = cfg->right_ascension, w1 = cfg->force_weight_to_one;
    const double max_w = cfg->max_w;
    auto record = [&](double f[6], int i) {
        if (ra) {
            f[0] *= -1.0;
            f[2] *= -1.0;
        }
        if (!w1) {
            f[3] *= f[5];
            f[4] *= f[5];
        }
        if ((double)std::fabs((float)f[2]) > max_w) f[2] = f[2] / (double)std::fabs((float)f[2]) * max_w;
        uvw[i].x = (float)(f[0] * m2w);
        uvw[i].y = (float)(f[1] * m2w);
        uvw[i].z = (float)(f[2] * m2w);
        vis[i].x = (float)f[3];
        vis[i].y = (float)f[4];
    };
    // records whose six fields are all in the file are independent
    const int full = (int)std::min<size_t>((size_t)n, t.size() / 6);
    {
        unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
        if (full < 100000) nt = 1;
        std::vector<std::thread> th;
        const int span = (full + (int)nt - 1) / (int)nt;
        auto work = [&](int b, int e) {
            for (int i = b; i < e; ++i) {
                double f[6];
                for (int k = 0; k < 6; ++k) f[k] = t[(size_t)6 * i + k];
                record(f, i);
            }
        };
        for (unsigned q = 0; q < nt; ++q) {
            const int b = std::min(full, (int)q * span), e = std::min(full, (int)(q + 1) * span);
            if (nt == 1) {
                work(b, e);
            } else {
                th.emplace_back(work, b, e);
            }
        }
        for (auto &x : th) x.join();
    }
    if (full < n) {
        // the rest of the loop with fscanf's stale variables (top.c:171-182):
        // state after the last full record, then the partial record's fields
        double f[6] = {0, 0, 0, 0, 0, 0};
        if (full > 0) {
            for (int k = 0; k < 6; ++k) f[k] = t[(size_t)6 * (full - 1) + k];
            if (ra) {
                f[0] *= -1.0;
                f[2] *= -1.0;
            }
            if (!w1) {
                f[3] *= f[5];
                f[4] *= f[5];
            }
            if ((double)std::fabs((float)f[2]) > max_w) f[2] = f[2] / (double)std::fabs((float)f[2]) * max_w;
        }
        for (int i = full; i < n; ++i) {
            for (int k = 0; k < 6; ++k) {
                const size_t idx = (size_t)6 * i + k;
                if (idx < t.size()) f[k] = t[idx];
            }
            record(f, i);
        }
    }
    return SDP_OK;
}

int load_psf(int G, int PG, const sdp_config *cfg, float *psf, double *psf_max)
{
    SDP_CHECK_ARG(G > 0 && PG > 0 && cfg && psf && psf_max, "bad argument");
    FileView buf;
    SDP_TRY(read_file(cfg->psf_input_file, buf));
    std::vector<double> t;
    parse_all(buf, 0, t);
    const size_t nfull = (size_t)PG * PG;
    std::vector<float> full(nfull, 0.f);
    double sample = 0.0;  // declared before the loop: stale once the file ends (top.c:476)
    for (size_t i = 0; i < nfull; ++i) {
        if (i < t.size()) sample = t[i];
        full[i] = (float)sample;
        if (sample > *psf_max) *psf_max = (float)sample;
    }
    std::memset(psf, 0, sizeof(float) * (size_t)G * G);
    const int smaller = std::min(PG, G);
    const int poff = std::max(0, (PG - G) / 2), goff = std::max(0, (G - PG) / 2);
    for (int y = 0; y < smaller; ++y)
        for (int x = 0; x < smaller; ++x)
            psf[(size_t)(y + goff) * G + (x + goff)] = full[(size_t)(y + poff) * PG + (x + poff)];
    for (size_t i = 0; i < (size_t)G * G; ++i) psf[i] = (float)((double)psf[i] / *psf_max);
    return SDP_OK;
}

}  // namespace

using sdp::actor_fail;

SDP_EXPORT void visibility_host_set_up(int NUM_VISIBILITIES, sdp_config *config, sdp_float3 *vis_uvw_coords,
                                       sdp_float2 *measured_vis)
{
    if (load_visibilities(NUM_VISIBILITIES, config, vis_uvw_coords, measured_vis) != SDP_OK)
        actor_fail("visibility_host_set_up");
}

SDP_EXPORT void kernel_host_set_up(int NUM_KERNELS, int TOTAL_KERNEL_SAMPLES, sdp_config *config,
                                   sdp_int2 *kernel_supports, sdp_float2 *kernels)
{
    (void)TOTAL_KERNEL_SAMPLES;
    if (!config || !kernel_supports || !kernels) {
        set_error(SDP_ERR_INVALID, "NULL argument");
        actor_fail("kernel_host_set_up");
        return;
    }
    if (load_kernels(config->kernel_support_file, config->kernel_real_file, config->kernel_imag_file, NUM_KERNELS,
                     config->oversampling, kernel_supports, kernels) != SDP_OK)
        actor_fail("kernel_host_set_up");
}

SDP_EXPORT void degridding_kernel_host_set_up(int NUM_KERNELS, int TOTAL_KERNEL_SAMPLES, sdp_config *config,
                                              sdp_int2 *degridding_kernel_supports, sdp_float2 *degridding_kernels)
{
    (void)TOTAL_KERNEL_SAMPLES;
    if (!config || !degridding_kernel_supports || !degridding_kernels) {
        set_error(SDP_ERR_INVALID, "NULL argument");
        actor_fail("degridding_kernel_host_set_up");
        return;
    }
    if (load_kernels(config->degridding_kernel_support_file, config->degridding_kernel_real_file,
                     config->degridding_kernel_imag_file, NUM_KERNELS, config->oversampling,
                     degridding_kernel_supports, degridding_kernels) != SDP_OK)
        actor_fail("degridding_kernel_host_set_up");
}

SDP_EXPORT void psf_host_set_up(int GRID_SIZE, int PSF_GRID_SIZE, sdp_config *config, float *psf,
                                double *psf_max_value)
{
    if (load_psf(GRID_SIZE, PSF_GRID_SIZE, config, psf, psf_max_value) != SDP_OK) actor_fail("psf_host_set_up");
}
