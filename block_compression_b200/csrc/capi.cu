// C ABI of the library (include/bc_capi.h): argument checks that mirror the
// reference's asserts, host<->device staging for the host-pointer entry
// points, and the GpuBlockCompressor-style task queue.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/bc_capi.h"
#include "bc_kernels.h"

namespace bcn {

static thread_local int t_last_cuda_error = 0;

static int cuda_fail(cudaError_t e) {
    t_last_cuda_error = (int)e;
    return BC_ERR_CUDA;
}
#define BC_CUDA(call)                              \
    do {                                           \
        cudaError_t e_ = (call);                   \
        if (e_ != cudaSuccess) return cuda_fail(e_); \
    } while (0)

static size_t block_bytes(int variant) { return (variant == BC_BC1 || variant == BC_BC4) ? 8 : 16; }

// Upper bounds for the search-effort knobs. The reference panics on partition
// thresholds above its list lengths (src/encode/bc7.rs:554, bc6h.rs:340); the
// iteration caps are this library's own guard against runaway launches.
static const uint32_t kMaxRefine = 64;

static int check_bc7(const void* p) {
    if (!p) return BC_ERR_NULL;
    const BC7SettingsDev* s = (const BC7SettingsDev*)p;
    if (s->channels != 3 && s->channels != 4) return BC_ERR_SETTINGS;
    if (s->fast_skip_threshold_mode1 > 64 || s->fast_skip_threshold_mode3 > 64 || s->fast_skip_threshold_mode7 > 64)
        return BC_ERR_SETTINGS;
    for (int i = 0; i < 8; i++)
        if (s->refine_iterations[i] > kMaxRefine) return BC_ERR_SETTINGS;
    if (s->refine_iterations_channel > kMaxRefine) return BC_ERR_SETTINGS;
    return BC_OK;
}

static int check_bc6h(const void* p) {
    if (!p) return BC_ERR_NULL;
    const BC6HSettingsDev* s = (const BC6HSettingsDev*)p;
    if (s->fast_skip_threshold > 32) return BC_ERR_SETTINGS;
    if (s->refine_iterations_1p > kMaxRefine || s->refine_iterations_2p > kMaxRefine) return BC_ERR_SETTINGS;
    return BC_OK;
}

// Entry points defined in other translation units share these checks.
int validate_bc7_settings(const void* p) { return check_bc7(p); }
void record_cuda_error(cudaError_t e) { t_last_cuda_error = (int)e; }

static int check_settings(int variant, const void* settings) {
    if (variant < 0 || variant > 6) return BC_ERR_VARIANT;
    if (variant == BC_BC7) return check_bc7(settings);
    if (variant == BC_BC6H) return check_bc6h(settings);
    return BC_OK;
}

// Per-device memory pool for the stream-ordered scratch of multi-kernel
// encodes. Its release threshold is unlimited, so memory freed at the end of
// one call is reused by the next instead of being unmapped at every
// synchronisation (the default pool's threshold is 0). The pool belongs to
// this library; the caller's default pool is left untouched.
static std::mutex g_pool_mu;
static cudaMemPool_t g_pools[64];

static int scratch_pool(cudaMemPool_t* out) {
    int dev = 0;
    BC_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return BC_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pools[dev]) {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool;
        BC_CUDA(cudaMemPoolCreate(&pool, &props));
        uint64_t threshold = UINT64_MAX;
        BC_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
        g_pools[dev] = pool;
    }
    *out = g_pools[dev];
    return BC_OK;
}

// Enqueues the encode of a w x h region whose row 0 is at `src`.
// bytes_per_px: 4 (RGBA8) or 8 (RGBA16F, BC6H only).
static int enqueue_encode(int variant, const void* settings, const uint8_t* src, size_t stride, uint32_t w,
                          uint32_t h, uint8_t* dst, int bc6h_source, cudaStream_t s) {
    uint32_t bw = (w + 3) / 4, bh = (h + 3) / 4;
    if (bw == 0 || bh == 0) return BC_OK;
    switch (variant) {
        case BC_BC7: {
            // Stream-ordered scratch from the library's pool: returned to the
            // pool once the launches have run.
            const BC7SettingsDev& s7 = *(const BC7SettingsDev*)settings;
            cudaMemPool_t pool;
            int prc = scratch_pool(&pool);
            if (prc != BC_OK) return prc;
            void* scratch = nullptr;
            BC_CUDA(cudaMallocFromPoolAsync(&scratch, bc7_scratch_bytes(bw * bh, s7), pool, s));
            cudaError_t e = launch_bc7_encode(src, stride, bw, bh, dst, s7, scratch, s);
            cudaError_t f = cudaFreeAsync(scratch, s);
            BC_CUDA(e);
            BC_CUDA(f);
            break;
        }
        case BC_BC6H: {
            int rc = upload_bc6h_tables();
            if (rc != BC_OK) return rc;
            const BC6HSettingsDev& s6 = *(const BC6HSettingsDev*)settings;
            cudaMemPool_t pool;
            rc = scratch_pool(&pool);
            if (rc != BC_OK) return rc;
            void* scratch = nullptr;
            BC_CUDA(cudaMallocFromPoolAsync(&scratch, bc6h_scratch_bytes(bw * bh, s6), pool, s));
            cudaError_t e = launch_bc6h_encode(src, stride, bc6h_source, bw, bh, dst, s6, scratch, s);
            cudaError_t f = cudaFreeAsync(scratch, s);
            BC_CUDA(e);
            BC_CUDA(f);
            break;
        }
        default:
            launch_bc15_encode(variant, src, stride, bw, bh, dst, s);
            break;
    }
    BC_CUDA(cudaGetLastError());
    return BC_OK;
}

// Per-thread device staging buffers for the host-pointer entry points.
struct Staging {
    void* buf[2] = {nullptr, nullptr};
    size_t cap[2] = {0, 0};
    int device = -1;
    ~Staging() {
        for (int i = 0; i < 2; i++)
            if (buf[i]) cudaFree(buf[i]);
    }
    int get(int i, size_t n, void** out) {
        int dev = 0;
        BC_CUDA(cudaGetDevice(&dev));
        if (dev != device) {
            for (int j = 0; j < 2; j++) {
                if (buf[j]) cudaFree(buf[j]);
                buf[j] = nullptr;
                cap[j] = 0;
            }
            device = dev;
        }
        if (cap[i] < n) {
            if (buf[i]) cudaFree(buf[i]);
            buf[i] = nullptr;
            cap[i] = 0;
            BC_CUDA(cudaMalloc(&buf[i], n));
            cap[i] = n;
        }
        *out = buf[i];
        return BC_OK;
    }
};
static thread_local Staging t_staging;

// ---- sRGB tables ---------------------------------------------------------------

// binary16 -> binary32 (exact)
static float half_bits_to_float(uint16_t h) {
    uint32_t sign = (uint32_t)(h >> 15) << 31, exp = (h >> 10) & 0x1F, man = h & 0x3FF, bits;
    if (exp == 0) {
        if (man == 0) {
            bits = sign;
        } else {
            int e = -1;
            do {
                e++;
                man <<= 1;
            } while ((man & 0x400) == 0);
            bits = sign | ((uint32_t)(127 - 15 - e) << 23) | ((man & 0x3FF) << 13);
        }
    } else if (exp == 31) {
        bits = sign | 0x7F800000u | (man << 13);
    } else {
        bits = sign | ((exp - 15 + 127) << 23) | (man << 13);
    }
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

// binary32 -> binary16, round to nearest even
static uint16_t float_to_half_bits(float f) {
    uint32_t x;
    memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u, exp = (x >> 23) & 0xFFu, man = x & 0x7FFFFFu;
    if (exp == 0xFF) return (uint16_t)(man ? (sign | 0x7E00u | (man >> 13)) : (sign | 0x7C00u));
    int e = (int)exp - 127 + 15;
    if (e >= 31) return (uint16_t)(sign | 0x7C00u);
    if (e <= 0) {
        if (e < -10) return (uint16_t)sign;
        uint32_t m = man | 0x800000u;
        int sh = 14 - e;
        uint32_t hm = m >> sh, rem = m & ((1u << sh) - 1), half = 1u << (sh - 1);
        if (rem > half || (rem == half && (hm & 1))) hm++;
        return (uint16_t)(sign | hm);
    }
    uint32_t hb = sign | ((uint32_t)e << 10) | (man >> 13), rem = man & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (hb & 1))) hb++;
    return (uint16_t)hb;
}

// Host-side evaluation of the reference's sRGB conversions with the C
// library's powf (what Rust's f32::powf calls on Linux), tabulated over every
// input the kernels can see.
static void build_srgb_tables(uint8_t* h2s, uint16_t* s2h) {
    for (int h = 0; h < 0x7C00; h++) {
        float lin = half_bits_to_float((uint16_t)h);  // decode.rs:151-159
        float v = lin <= 0.0031308f ? lin * 12.92f : 1.055f * powf(lin, 1.0f / 2.4f) - 0.055f;
        if (v < 0.0f) v = 0.0f;
        if (v > 1.0f) v = 1.0f;
        float r = roundf(v * 255.0f);
        h2s[h] = std::isnan(r) ? 0 : (uint8_t)r;
    }
    for (int s = 0; s < 256; s++) {  // bc6h.rs:20-27, then half::f16::from_f32
        float v = (float)s / 255.0f;
        float lin = v <= 0.04045f ? v / 12.92f : powf((v + 0.055f) / 1.055f, 2.4f);
        s2h[s] = float_to_half_bits(lin);
    }
}

static std::mutex g_table_mu;
static bool g_tables_ready[64];

int upload_bc6h_tables() {
    int dev = 0;
    BC_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return BC_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_table_mu);
    if (g_tables_ready[dev]) return BC_OK;
    static uint8_t h2s[0x7C00];
    static uint16_t s2h[256];
    static bool built = false;
    if (!built) {
        build_srgb_tables(h2s, s2h);
        built = true;
    }
    BC_CUDA(set_half_to_srgb_table(h2s));
    BC_CUDA(set_srgb_to_half_table(s2h));
    g_tables_ready[dev] = true;
    return BC_OK;
}

}  // namespace bcn

using namespace bcn;

// ---- presets (src/settings.rs:217-441) ----------------------------------------------

extern "C" int bc_bc6h_settings_preset(const char* name, bc_bc6h_settings* out) {
    if (!name || !out) return BC_ERR_NULL;
    struct P {
        const char* n;
        bc_bc6h_settings s;
    };
    static const P presets[] = {
        {"very_fast", {0, 1, 0, 0, 0}}, {"fast", {0, 1, 0, 1, 2}}, {"basic", {0, 0, 2, 2, 4}},
        {"slow", {1, 0, 2, 2, 10}},     {"very_slow", {1, 0, 2, 2, 32}},
    };
    for (const P& p : presets)
        if (strcmp(p.n, name) == 0) {
            *out = p.s;
            return BC_OK;
        }
    return BC_ERR_SETTINGS;
}

extern "C" int bc_bc7_settings_preset(const char* name, bc_bc7_settings* out) {
    if (!name || !out) return BC_ERR_NULL;
    struct P {
        const char* n;
        bc_bc7_settings s;
    };
    // {refine_iterations[8]}, {mode_selection[4]}, skip_mode2, t1, t3, t7, mode45_channel0, refine_channel, channels
    static const P presets[] = {
        {"opaque_ultra_fast", {{2, 2, 2, 1, 2, 2, 1, 0}, {0, 0, 0, 1}, 1, 3, 1, 0, 0, 0, 3}},
        {"opaque_very_fast", {{2, 2, 2, 1, 2, 2, 1, 0}, {0, 1, 0, 1}, 1, 3, 1, 0, 0, 0, 3}},
        {"opaque_fast", {{2, 2, 2, 1, 2, 2, 2, 0}, {0, 1, 0, 1}, 1, 12, 4, 0, 0, 0, 3}},
        {"opaque_basic", {{2, 2, 2, 2, 2, 2, 2, 0}, {1, 1, 1, 1}, 1, 12, 8, 0, 0, 2, 3}},
        {"opaque_slow", {{4, 4, 4, 4, 4, 4, 4, 0}, {1, 1, 1, 1}, 0, 64, 64, 0, 0, 4, 3}},
        {"alpha_ultrafast", {{2, 1, 2, 1, 1, 1, 2, 2}, {0, 0, 1, 1}, 1, 0, 0, 4, 3, 1, 4}},
        {"alpha_very_fast", {{2, 1, 2, 1, 2, 2, 2, 2}, {0, 1, 1, 1}, 1, 0, 0, 4, 3, 2, 4}},
        {"alpha_fast", {{2, 1, 2, 1, 2, 2, 2, 2}, {0, 1, 1, 1}, 1, 4, 4, 8, 3, 2, 4}},
        {"alpha_basic", {{2, 2, 2, 2, 2, 2, 2, 2}, {1, 1, 1, 1}, 1, 12, 8, 8, 0, 2, 4}},
        {"alpha_slow", {{4, 4, 4, 4, 4, 4, 4, 4}, {1, 1, 1, 1}, 0, 64, 64, 64, 0, 4, 4}},
    };
    for (const P& p : presets)
        if (strcmp(p.n, name) == 0) {
            *out = p.s;
            return BC_OK;
        }
    return BC_ERR_SETTINGS;
}

// ---- sizes (src/lib.rs:129-157) ---------------------------------------------------------

extern "C" uint32_t bc_bytes_per_row(int variant, uint32_t width) {
    if (variant < 0 || variant > 6) return 0;
    return ((width + 3) / 4) * (uint32_t)block_bytes(variant);
}

extern "C" size_t bc_blocks_byte_size(int variant, uint32_t width, uint32_t height) {
    if (variant < 0 || variant > 6) return 0;
    return ((size_t)(width + 3) / 4) * ((size_t)(height + 3) / 4) * block_bytes(variant);
}

// ---- encode ------------------------------------------------------------------------------

// src/encode.rs:91-101 plus the source-extent check the Rust slice indexing does.
static int check_encode(int variant, const void* settings, size_t src_len, size_t blocks_len, uint32_t w, uint32_t h,
                        size_t stride_bytes, size_t bytes_per_px) {
    if (h % 4 != 0 || w % 4 != 0) return BC_ERR_DIMS;
    int rc = check_settings(variant, settings);
    if (rc != BC_OK) return rc;
    if (blocks_len < bc_blocks_byte_size(variant, w, h)) return BC_ERR_DST_SIZE;
    if (w > 0 && h > 0 && src_len < (size_t)(h - 1) * stride_bytes + (size_t)w * bytes_per_px) return BC_ERR_SRC_SIZE;
    return BC_OK;
}

extern "C" int bc_compress_rgba8_device(int variant, const void* settings, const uint8_t* rgba_dev, size_t rgba_len,
                                        uint8_t* blocks_dev, size_t blocks_len, uint32_t width, uint32_t height,
                                        size_t stride_bytes, void* stream) {
    int rc = check_encode(variant, settings, rgba_len, blocks_len, width, height, stride_bytes, 4);
    if (rc != BC_OK) return rc;
    if (width == 0 || height == 0) return BC_OK;
    if (!rgba_dev || !blocks_dev) return BC_ERR_NULL;
    return enqueue_encode(variant, settings, rgba_dev, stride_bytes, width, height, blocks_dev, BC6H_SRC_RGBA8_SRGB,
                          (cudaStream_t)stream);
}

extern "C" int bc_compress_rgba16_device(const bc_bc6h_settings* settings, const uint16_t* rgba_dev, size_t rgba_len,
                                         uint8_t* blocks_dev, size_t blocks_len, uint32_t width, uint32_t height,
                                         size_t stride_elems, void* stream) {
    int rc = check_encode(BC_BC6H, settings, rgba_len * 2, blocks_len, width, height, stride_elems * 2, 8);
    if (rc != BC_OK) return rc;
    if (width == 0 || height == 0) return BC_OK;
    if (!rgba_dev || !blocks_dev) return BC_ERR_NULL;
    return enqueue_encode(BC_BC6H, settings, (const uint8_t*)rgba_dev, stride_elems * 2, width, height, blocks_dev,
                          BC6H_SRC_RGBA16F, (cudaStream_t)stream);
}

// Streams and events of the pipelined host-buffer encode, per thread and
// device (created on first use).
struct HostPipe {
    static constexpr int kRing = 4;
    cudaStream_t up = nullptr, comp = nullptr, down = nullptr;
    cudaEvent_t ev_up[kRing] = {}, ev_comp[kRing] = {};
    int device = -1;
    void release() {
        for (int i = 0; i < kRing; i++) {
            if (ev_up[i]) cudaEventDestroy(ev_up[i]);
            if (ev_comp[i]) cudaEventDestroy(ev_comp[i]);
            ev_up[i] = ev_comp[i] = nullptr;
        }
        for (cudaStream_t* st : {&up, &comp, &down})
            if (*st) {
                cudaStreamDestroy(*st);
                *st = nullptr;
            }
        device = -1;
    }
    ~HostPipe() { release(); }
    int get() {
        int dev = 0;
        BC_CUDA(cudaGetDevice(&dev));
        if (dev == device) return BC_OK;
        release();
        for (cudaStream_t* st : {&up, &comp, &down}) BC_CUDA(cudaStreamCreateWithFlags(st, cudaStreamNonBlocking));
        for (int i = 0; i < kRing; i++) {
            BC_CUDA(cudaEventCreateWithFlags(&ev_up[i], cudaEventDisableTiming));
            BC_CUDA(cudaEventCreateWithFlags(&ev_comp[i], cudaEventDisableTiming));
        }
        device = dev;
        return BC_OK;
    }
};
static thread_local HostPipe t_pipe;

// One band of host_encode: rows y0 .. y0 + h - 1 up, encoded, blocks down.
static int enqueue_band(int variant, const void* settings, const uint8_t* src, uint8_t* dsrc, size_t stride_bytes,
                        size_t bpp, uint8_t* blocks, uint8_t* ddst, uint32_t width, uint32_t y0, uint32_t h,
                        size_t block_row_bytes, int bc6h_source, int ring) {
    const size_t soff = (size_t)y0 * stride_bytes;
    const size_t sbytes = (size_t)(h - 1) * stride_bytes + (size_t)width * bpp;
    const size_t doff = (size_t)(y0 / 4) * block_row_bytes;
    const size_t dbytes = (size_t)((h + 3) / 4) * block_row_bytes;
    cudaEvent_t eu = t_pipe.ev_up[ring], ec = t_pipe.ev_comp[ring];
    BC_CUDA(cudaMemcpyAsync(dsrc + soff, src + soff, sbytes, cudaMemcpyHostToDevice, t_pipe.up));
    BC_CUDA(cudaEventRecord(eu, t_pipe.up));
    BC_CUDA(cudaStreamWaitEvent(t_pipe.comp, eu, 0));
    int rc = enqueue_encode(variant, settings, dsrc + soff, stride_bytes, width, h, ddst + doff, bc6h_source,
                            t_pipe.comp);
    if (rc != BC_OK) return rc;
    BC_CUDA(cudaEventRecord(ec, t_pipe.comp));
    BC_CUDA(cudaStreamWaitEvent(t_pipe.down, ec, 0));
    BC_CUDA(cudaMemcpyAsync(blocks + doff, ddst + doff, dbytes, cudaMemcpyDeviceToHost, t_pipe.down));
    return BC_OK;
}

// Source bytes of the first band and of the later ones of a host-buffer
// encode (whole block rows, rounded down). On the benchmark's four 2048x2048
// textures called one after another, 2 + 8 MiB bands measured 1% faster than
// 4 + 4 MiB, 1 + 2 MiB 8% slower (fewer, larger BC7 launches win; the shorter
// first upload gains less).
#ifndef BCN_FIRST_BAND_KIB
#define BCN_FIRST_BAND_KIB 2048
#endif
#ifndef BCN_BAND_KIB
#define BCN_BAND_KIB 8192
#endif

// Host-buffer encode, pipelined: the image is cut into bands of whole block
// rows (about 2 MiB of source for the first, 8 MiB for the others) and band
// i's upload, encode and download run on three streams, so the copies of one
// band overlap the kernels of its neighbours. Blocks are independent and every band but the last is a whole
// number of block rows, so the bands' blocks are exactly the image's.
static int host_encode(int variant, const void* settings, const uint8_t* src, size_t stride_bytes, size_t bpp,
                       uint8_t* blocks, uint32_t width, uint32_t height, int bc6h_source) {
    size_t src_bytes = (size_t)(height - 1) * stride_bytes + (size_t)width * bpp;
    size_t dst_bytes = bc_blocks_byte_size(variant, width, height);
    void *dsrc = nullptr, *ddst = nullptr;
    int rc = t_staging.get(0, src_bytes, &dsrc);
    if (rc != BC_OK) return rc;
    rc = t_staging.get(1, dst_bytes, &ddst);
    if (rc != BC_OK) return rc;
    rc = t_pipe.get();
    if (rc != BC_OK) return rc;
    const size_t block_row_bytes = bc_blocks_byte_size(variant, width, 4);
    // whole block rows of about `target` source bytes (at least one)
    auto rows_for = [&](size_t target) {
        uint32_t r = (uint32_t)(target / (stride_bytes ? stride_bytes : 1)) & ~3u;
        return r < 4 ? 4u : r;
    };
    // The first band is smaller, so the first encode starts after a short
    // upload; the later bands' uploads hide behind the encodes before them.
    const uint32_t first_rows = rows_for((size_t)BCN_FIRST_BAND_KIB << 10), band_rows = rows_for((size_t)BCN_BAND_KIB << 10);
    int brc = BC_OK;
    uint32_t b = 0;
    for (uint32_t y0 = 0; y0 < height && brc == BC_OK; b++) {
        const uint32_t rows = b == 0 ? first_rows : band_rows;
        const uint32_t h = height - y0 < rows ? height - y0 : rows;
        brc = enqueue_band(variant, settings, src, (uint8_t*)dsrc, stride_bytes, bpp, blocks, (uint8_t*)ddst, width,
                           y0, h, block_row_bytes, bc6h_source, b % HostPipe::kRing);
        y0 += h;
    }
    // every band's copies have finished before the caller's buffers are
    // released, on the error path too
    cudaError_t e0 = cudaStreamSynchronize(t_pipe.up);
    cudaError_t e1 = cudaStreamSynchronize(t_pipe.comp);
    cudaError_t e2 = cudaStreamSynchronize(t_pipe.down);
    if (brc != BC_OK) return brc;
    BC_CUDA(e0);
    BC_CUDA(e1);
    BC_CUDA(e2);
    return BC_OK;
}

extern "C" int bc_compress_rgba8(int variant, const void* settings, const uint8_t* rgba, size_t rgba_len,
                                 uint8_t* blocks, size_t blocks_len, uint32_t width, uint32_t height, uint32_t stride) {
    int rc = check_encode(variant, settings, rgba_len, blocks_len, width, height, stride, 4);
    if (rc != BC_OK) return rc;
    if (width == 0 || height == 0) return BC_OK;
    if (!rgba || !blocks) return BC_ERR_NULL;
    return host_encode(variant, settings, rgba, stride, 4, blocks, width, height, BC6H_SRC_RGBA8_SRGB);
}

extern "C" int bc_compress_rgba16(int variant, const bc_bc6h_settings* settings, const uint16_t* rgba, size_t rgba_len,
                                  uint8_t* blocks, size_t blocks_len, uint32_t width, uint32_t height,
                                  uint32_t stride) {
    if (variant != BC_BC6H) return BC_ERR_VARIANT;  // src/encode.rs:247-249
    int rc = check_encode(BC_BC6H, settings, rgba_len * 2, blocks_len, width, height, (size_t)stride * 2, 8);
    if (rc != BC_OK) return rc;
    if (width == 0 || height == 0) return BC_OK;
    if (!rgba || !blocks) return BC_ERR_NULL;
    return host_encode(BC_BC6H, settings, (const uint8_t*)rgba, (size_t)stride * 2, 8, blocks, width, height,
                       BC6H_SRC_RGBA16F);
}

// ---- decode (src/decode.rs:336-468) -------------------------------------------------------

// out_format: 0 RGBA8, 1 RGBA16F, 2 RGBA32F. Checks of decode.rs:343-355 and
// :404-417; any dimension that is not a multiple of 4 makes the reference
// write past its output slice and panic.
static int check_decode(int variant, uint32_t w, uint32_t h, size_t blocks_len, size_t out_len, int out_format) {
    if (variant < 0 || variant > 6) return BC_ERR_VARIANT;
    if (out_format != 0 && variant != BC_BC6H) return BC_ERR_VARIANT;  // decode.rs:423-426
    if (out_format < 0 || out_format > 2) return BC_ERR_VARIANT;
    if (blocks_len != bc_blocks_byte_size(variant, w, h)) return BC_ERR_SRC_SIZE;
    if (out_len != (size_t)w * h * 4) return BC_ERR_DST_SIZE;
    if (w % 4 != 0 || h % 4 != 0) return BC_ERR_DIMS;
    return BC_OK;
}

static int enqueue_decode(int variant, uint32_t w, uint32_t h, const uint8_t* blocks, void* out, int fmt,
                          cudaStream_t s) {
    uint32_t bw = (w + 3) / 4, bh = (h + 3) / 4;
    if (bw == 0 || bh == 0) return BC_OK;
    size_t pitch = (size_t)w * 4;  // elements of the output type
    if (variant == BC_BC7) {
        launch_bc7_decode(blocks, bw, bh, (uint8_t*)out, pitch, s);
    } else if (variant == BC_BC6H) {
        int rc = upload_bc6h_tables();
        if (rc != BC_OK) return rc;
        launch_bc6h_decode(blocks, bw, bh, out, pitch, fmt, s);
    } else {
        launch_bc15_decode(variant, blocks, bw, bh, (uint8_t*)out, pitch, s);
    }
    BC_CUDA(cudaGetLastError());
    return BC_OK;
}

extern "C" int bc_decompress_device(int variant, uint32_t width, uint32_t height, const uint8_t* blocks_dev,
                                    size_t blocks_len, void* out_dev, size_t out_len, int out_format, void* stream) {
    int rc = check_decode(variant, width, height, blocks_len, out_len, out_format);
    if (rc != BC_OK) return rc;
    if (width == 0 || height == 0) return BC_OK;
    if (!blocks_dev || !out_dev) return BC_ERR_NULL;
    return enqueue_decode(variant, width, height, blocks_dev, out_dev, out_format, (cudaStream_t)stream);
}

static int host_decode(int variant, uint32_t w, uint32_t h, const uint8_t* blocks, size_t blocks_len, void* out,
                       size_t out_len, int fmt) {
    int rc = check_decode(variant, w, h, blocks_len, out_len, fmt);
    if (rc != BC_OK) return rc;
    if (w == 0 || h == 0) return BC_OK;
    if (!blocks || !out) return BC_ERR_NULL;
    size_t esz = fmt == 0 ? 1 : (fmt == 1 ? 2 : 4);
    size_t out_bytes = out_len * esz;
    void *dsrc = nullptr, *ddst = nullptr;
    rc = t_staging.get(0, blocks_len, &dsrc);
    if (rc != BC_OK) return rc;
    rc = t_staging.get(1, out_bytes, &ddst);
    if (rc != BC_OK) return rc;
    cudaStream_t s = 0;
    BC_CUDA(cudaMemcpyAsync(dsrc, blocks, blocks_len, cudaMemcpyHostToDevice, s));
    // The BC6H float layouts leave 4 elements per block row untouched; carry the
    // caller's values through so the untouched elements keep them, as in the
    // reference.
    if (fmt != 0) BC_CUDA(cudaMemcpyAsync(ddst, out, out_bytes, cudaMemcpyHostToDevice, s));
    rc = enqueue_decode(variant, w, h, (const uint8_t*)dsrc, ddst, fmt, s);
    if (rc != BC_OK) return rc;
    BC_CUDA(cudaMemcpyAsync(out, ddst, out_bytes, cudaMemcpyDeviceToHost, s));
    BC_CUDA(cudaStreamSynchronize(s));
    return BC_OK;
}

extern "C" int bc_decompress_blocks_as_rgba8(int variant, uint32_t width, uint32_t height, const uint8_t* blocks,
                                             size_t blocks_len, uint8_t* rgba, size_t rgba_len) {
    return host_decode(variant, width, height, blocks, blocks_len, rgba, rgba_len, 0);
}

extern "C" int bc_decompress_blocks_as_rgba16f(int variant, uint32_t width, uint32_t height, const uint8_t* blocks,
                                               size_t blocks_len, uint16_t* rgba, size_t rgba_len) {
    if (variant != BC_BC6H) return BC_ERR_VARIANT;
    return host_decode(variant, width, height, blocks, blocks_len, rgba, rgba_len, 1);
}

extern "C" int bc_decompress_blocks_as_rgba32f(int variant, uint32_t width, uint32_t height, const uint8_t* blocks,
                                               size_t blocks_len, float* rgba, size_t rgba_len) {
    if (variant != BC_BC6H) return BC_ERR_VARIANT;
    return host_decode(variant, width, height, blocks, blocks_len, rgba, rgba_len, 2);
}

// ---- per-block decoders (src/decode/block.rs:50-119, 262, 774, 801) --------------------------

// Bytes one compressed block of `kind` occupies, and the element size of its output.
static size_t block_kind_bytes(int kind) { return (kind == BC_BLOCK_BC1 || kind == BC_BLOCK_BC4) ? 8 : 16; }
static size_t block_kind_elem(int kind) {
    return kind == BC_BLOCK_BC6H ? 2 : (kind == BC_BLOCK_BC6H_FLOAT ? 4 : 1);
}

// Output elements the reference's slice indexing needs (it panics on
// less): one past the last element written, and for the BC6H float form also
// 4 * pitch, because it advances its output slice by the pitch after each of
// the 4 rows (block.rs:789-795).
extern "C" size_t bc_decode_block_min_len(int kind, size_t pitch) {
    switch (kind) {
        case BC_BLOCK_BC1: case BC_BLOCK_BC2: case BC_BLOCK_BC3: case BC_BLOCK_BC7: return 3 * pitch + 16;
        case BC_BLOCK_BC4: return 3 * pitch + 4;
        case BC_BLOCK_BC5: return 3 * pitch + 8;
        case BC_BLOCK_BC6H: return 3 * pitch + 12;
        case BC_BLOCK_BC6H_FLOAT: return 4 * pitch > 3 * pitch + 12 ? 4 * pitch : 3 * pitch + 12;
        default: return 0;
    }
}

static int internal_block_kind(int kind, int is_signed) {
    if (kind == BC_BLOCK_BC6H) return is_signed ? BLOCK_BC6H_HALF_SIGNED : BLOCK_BC6H_HALF;
    if (kind == BC_BLOCK_BC6H_FLOAT) return is_signed ? BLOCK_BC6H_FLOAT_SIGNED : BLOCK_BC6H_FLOAT;
    return kind;
}

static int check_block_decode(int kind, int is_signed, size_t nblocks, size_t out_len, size_t pitch,
                              size_t out_block_stride) {
    if (kind < BC_BLOCK_BC1 || kind > BC_BLOCK_BC7) return BC_ERR_VARIANT;
    if (is_signed && kind != BC_BLOCK_BC6H && kind != BC_BLOCK_BC6H_FLOAT) return BC_ERR_VARIANT;
    if (nblocks == 0) return BC_OK;
    const size_t need = bc_decode_block_min_len(kind, pitch);
    if (nblocks > 1 && out_block_stride > (SIZE_MAX - need) / (nblocks - 1)) return BC_ERR_DST_SIZE;
    if (out_len < (nblocks - 1) * out_block_stride + need) return BC_ERR_DST_SIZE;
    return BC_OK;
}

extern "C" int bc_decode_blocks_device(int kind, int is_signed, const uint8_t* blocks_dev, size_t nblocks,
                                       void* out_dev, size_t out_len, size_t pitch, size_t out_block_stride,
                                       void* stream) {
    int rc = check_block_decode(kind, is_signed, nblocks, out_len, pitch, out_block_stride);
    if (rc != BC_OK || nblocks == 0) return rc;
    if (!blocks_dev || !out_dev) return BC_ERR_NULL;
    launch_decode_blocks(internal_block_kind(kind, is_signed), blocks_dev, nblocks, out_dev, pitch,
                         out_block_stride, (cudaStream_t)stream);
    BC_CUDA(cudaGetLastError());
    return BC_OK;
}

// One block from host memory: staged through the device (the output's
// current contents are carried through, since the reference leaves every
// element it does not write untouched), decoded, copied back; synchronous.
static int host_decode_block(int kind, int is_signed, const uint8_t* compressed, size_t compressed_len, void* out,
                             size_t out_len, size_t pitch) {
    int rc = check_block_decode(kind, is_signed, 1, out_len, pitch, 0);
    if (rc != BC_OK) return rc;
    if (!compressed || !out) return BC_ERR_NULL;
    const size_t nb = block_kind_bytes(kind);
    if (compressed_len < nb) return BC_ERR_SRC_SIZE;
    const size_t bytes = bc_decode_block_min_len(kind, pitch) * block_kind_elem(kind);
    void *dsrc = nullptr, *ddst = nullptr;
    rc = t_staging.get(0, nb, &dsrc);
    if (rc != BC_OK) return rc;
    rc = t_staging.get(1, bytes, &ddst);
    if (rc != BC_OK) return rc;
    cudaStream_t s = 0;
    BC_CUDA(cudaMemcpyAsync(dsrc, compressed, nb, cudaMemcpyHostToDevice, s));
    BC_CUDA(cudaMemcpyAsync(ddst, out, bytes, cudaMemcpyHostToDevice, s));
    launch_decode_blocks(internal_block_kind(kind, is_signed), (const uint8_t*)dsrc, 1, ddst, pitch, 0, s);
    BC_CUDA(cudaGetLastError());
    BC_CUDA(cudaMemcpyAsync(out, ddst, bytes, cudaMemcpyDeviceToHost, s));
    BC_CUDA(cudaStreamSynchronize(s));
    return BC_OK;
}

extern "C" int bc_decode_block_bc1(const uint8_t* compressed_block, size_t compressed_len, uint8_t* decompressed_block,
                                   size_t decompressed_len, size_t destination_pitch) {
    return host_decode_block(BC_BLOCK_BC1, 0, compressed_block, compressed_len, decompressed_block, decompressed_len,
                             destination_pitch);
}
extern "C" int bc_decode_block_bc2(const uint8_t* compressed_block, size_t compressed_len, uint8_t* decompressed_block,
                                   size_t decompressed_len, size_t destination_pitch) {
    return host_decode_block(BC_BLOCK_BC2, 0, compressed_block, compressed_len, decompressed_block, decompressed_len,
                             destination_pitch);
}
extern "C" int bc_decode_block_bc3(const uint8_t* compressed_block, size_t compressed_len, uint8_t* decompressed_block,
                                   size_t decompressed_len, size_t destination_pitch) {
    return host_decode_block(BC_BLOCK_BC3, 0, compressed_block, compressed_len, decompressed_block, decompressed_len,
                             destination_pitch);
}
extern "C" int bc_decode_block_bc4(const uint8_t* compressed_block, size_t compressed_len, uint8_t* decompressed_block,
                                   size_t decompressed_len, size_t destination_pitch) {
    return host_decode_block(BC_BLOCK_BC4, 0, compressed_block, compressed_len, decompressed_block, decompressed_len,
                             destination_pitch);
}
extern "C" int bc_decode_block_bc5(const uint8_t* compressed_block, size_t compressed_len, uint8_t* decompressed_block,
                                   size_t decompressed_len, size_t destination_pitch) {
    return host_decode_block(BC_BLOCK_BC5, 0, compressed_block, compressed_len, decompressed_block, decompressed_len,
                             destination_pitch);
}
extern "C" int bc_decode_block_bc6h(const uint8_t* compressed_block, size_t compressed_len,
                                    uint16_t* decompressed_block, size_t decompressed_len, size_t destination_pitch,
                                    int is_signed) {
    return host_decode_block(BC_BLOCK_BC6H, is_signed, compressed_block, compressed_len, decompressed_block,
                             decompressed_len, destination_pitch);
}
extern "C" int bc_decode_block_bc6h_float(const uint8_t* compressed_block, size_t compressed_len,
                                          float* decompressed_block, size_t decompressed_len, size_t destination_pitch,
                                          int is_signed) {
    return host_decode_block(BC_BLOCK_BC6H_FLOAT, is_signed, compressed_block, compressed_len, decompressed_block,
                             decompressed_len, destination_pitch);
}
extern "C" int bc_decode_block_bc7(const uint8_t* compressed_block, size_t compressed_len, uint8_t* decompressed_block,
                                   size_t decompressed_len, size_t destination_pitch) {
    return host_decode_block(BC_BLOCK_BC7, 0, compressed_block, compressed_len, decompressed_block, decompressed_len,
                             destination_pitch);
}

// ---- task queue (src/block_compressor.rs:44-590) --------------------------------------------

struct BcTask {
    int variant;
    BC7SettingsDev s7;
    BC6HSettingsDev s6;
    const uint8_t* src;   // row 0 of the region (texture_y_offset applied)
    size_t pitch;
    uint32_t w, h;
    uint8_t* dst;         // first block of the region (blocks_offset applied)
};

struct bc_compressor {
    int device;
    std::vector<BcTask> tasks;
};

extern "C" int bc_compressor_create(int device, bc_compressor** out) {
    if (!out) return BC_ERR_NULL;
    int count = 0;
    BC_CUDA(cudaGetDeviceCount(&count));
    if (count == 0) return BC_ERR_NO_DEVICE;
    if (device < 0) BC_CUDA(cudaGetDevice(&device));
    if (device >= count) return BC_ERR_NO_DEVICE;
    bc_compressor* c = new bc_compressor();
    c->device = device;
    *out = c;
    return BC_OK;
}

extern "C" int bc_compressor_destroy(bc_compressor* c) {
    delete c;
    return BC_OK;
}

extern "C" int bc_compressor_task_count(const bc_compressor* c) { return c ? (int)c->tasks.size() : 0; }

extern "C" int bc_compressor_add_task(bc_compressor* c, int variant, const void* settings, const void* src_dev,
                                      size_t src_pitch, size_t src_len, uint32_t width, uint32_t height,
                                      uint32_t texture_y_offset, void* dst_dev, size_t dst_len,
                                      uint32_t blocks_offset) {
    if (!c) return BC_ERR_TASKS;
    // block_compressor.rs:352-373
    if (height % 4 != 0 || width % 4 != 0 || texture_y_offset % 4 != 0) return BC_ERR_DIMS;
    int rc = check_settings(variant, settings);
    if (rc != BC_OK) return rc;
    size_t required = bc_blocks_byte_size(variant, width, height);
    if (dst_len < (size_t)blocks_offset + required) return BC_ERR_DST_SIZE;
    size_t bpp = variant == BC_BC6H ? 8 : 4;
    if (width > 0 && height > 0 &&
        src_len < (size_t)(texture_y_offset + height - 1) * src_pitch + (size_t)width * bpp)
        return BC_ERR_SRC_SIZE;
    if (width > 0 && height > 0 && (!src_dev || !dst_dev)) return BC_ERR_NULL;
    if (c->tasks.size() >= (1u << 20)) return BC_ERR_TASKS;
    BcTask t;
    memset(&t, 0, sizeof(t));
    t.variant = variant;
    if (variant == BC_BC7) t.s7 = *(const BC7SettingsDev*)settings;
    if (variant == BC_BC6H) t.s6 = *(const BC6HSettingsDev*)settings;
    t.src = (const uint8_t*)src_dev + (size_t)texture_y_offset * src_pitch;
    t.pitch = src_pitch;
    t.w = width;
    t.h = height;
    // The reference addresses the buffer in u32 words (blocks_offset / 4,
    // block_compressor.rs:449).
    t.dst = (uint8_t*)dst_dev + (blocks_offset & ~3u);
    c->tasks.push_back(t);
    return BC_OK;
}

extern "C" int bc_compressor_compress(bc_compressor* c, void* stream) {
    if (!c) return BC_ERR_TASKS;
    int prev = 0;
    BC_CUDA(cudaGetDevice(&prev));
    if (prev != c->device) BC_CUDA(cudaSetDevice(c->device));
    int rc = BC_OK;
    for (const BcTask& t : c->tasks) {
        const void* s = t.variant == BC_BC7 ? (const void*)&t.s7 : (const void*)&t.s6;
        rc = enqueue_encode(t.variant, s, t.src, t.pitch, t.w, t.h, t.dst, BC6H_SRC_RGBA16F, (cudaStream_t)stream);
        if (rc != BC_OK) break;
    }
    c->tasks.clear();
    if (prev != c->device) cudaSetDevice(prev);
    return rc;
}

// Task access for the batched path (batch.cu).
namespace bcn {
struct BcTaskView {
    int variant;
    const void* settings;
    const uint8_t* src;
    size_t pitch;
    uint32_t w, h;
    uint8_t* dst;
};
int compressor_tasks(bc_compressor* c, std::vector<BcTaskView>& out, int* device) {
    if (!c) return BC_ERR_TASKS;
    *device = c->device;
    out.clear();
    for (const BcTask& t : c->tasks) {
        BcTaskView v;
        v.variant = t.variant;
        v.settings = t.variant == BC_BC7 ? (const void*)&t.s7 : (const void*)&t.s6;
        v.src = t.src;
        v.pitch = t.pitch;
        v.w = t.w;
        v.h = t.h;
        v.dst = t.dst;
        out.push_back(v);
    }
    return BC_OK;
}
void compressor_clear(bc_compressor* c) {
    if (c) c->tasks.clear();
}
}  // namespace bcn

// ---- diagnostics ------------------------------------------------------------------------------

extern "C" int bc_last_cuda_error(void) { return t_last_cuda_error; }

extern "C" int bc_check_enabled(void) {
#ifdef BCN_CHECK
    return 1;
#else
    return 0;
#endif
}

extern "C" int bc_check_read(uint64_t out[3]) {
    if (!out) return BC_ERR_NULL;
    out[0] = out[1] = out[2] = 0;
    cudaError_t (*const take[])(unsigned long long*) = {check_take_bc7, check_take_bc6h, check_take_bc15,
                                                        check_take_decode};
    for (auto f : take) {
        unsigned long long r[3];
        BC_CUDA(f(r));
        if (r[0] != 0 && out[0] == 0) {
            out[0] = r[0] - 1;  // site
            out[1] = r[1];
            out[2] = r[2];
        }
    }
    return BC_OK;
}

extern "C" int bc_check_selftest(uint64_t index, uint64_t extent, void* stream) {
    BC_CUDA(launch_check_selftest(index, extent, (cudaStream_t)stream));
    return BC_OK;
}

extern "C" const char* bc_version(void) { return "bcn-b200 0.1.0 (sm_100a)"; }
