// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle_common.h, oracle_count.h).
// Entry points of the op-counting build: per-block op counts of the
// reference encoders.
#include <cstdint>
#include <cstring>

#include "oracle_common.h"

namespace oracle {
thread_local uint64_t g_ops = 0;
}

using namespace oracle;

static void to_real(const float* in, real* out) {
    for (int i = 0; i < 64; i++) out[i] = real(in[i]);
}

extern "C" uint64_t oracle_count_bc7(const float* block, const void* settings) {
    real b[64];
    to_real(block, b);
    uint32_t out[4];
    g_ops = 0;
    bc7_encode_block(b, (const BC7Settings*)settings, out);
    return g_ops;
}

extern "C" uint64_t oracle_count_bc6h(const float* block, const void* settings) {
    real b[64];
    to_real(block, b);
    uint32_t out[4];
    g_ops = 0;
    bc6h_encode_block(b, (const BC6HSettings*)settings, out);
    return g_ops;
}

extern "C" uint64_t oracle_count_bc1(const float* block) {
    real b[64];
    to_real(block, b);
    uint32_t out[2];
    g_ops = 0;
    bc1_core(b, out);
    return g_ops;
}

extern "C" uint64_t oracle_count_bc3_alpha(const float* block) {
    real b[64];
    to_real(block, b);
    uint32_t out[2];
    g_ops = 0;
    bc3_alpha(b, out);
    return g_ops;
}
