// Bounds-checked debug build of the kernels.
//
// Built with -DBCN_CHECK (build.py's check variant, libbcn_b200_check.so),
// every guarded index is compared with the extent of the array it indexes
// before the access: source rows and columns of the staged tiles, the rows and
// blocks of the per-block scratch arrays, the output blocks, and the
// shared-memory slots of the sorting decoders. A failed guard records
// (site, index, extent) in its translation unit's check record -- the first
// failure wins -- and the access is skipped (a load yields a neutral value).
// Nothing traps or asserts, so the context stays usable; the host reads and
// clears the records with bc_check_read(). Without BCN_CHECK the guards are
// the constant `true` and compile to nothing.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace bcn {

// Guard sites (the value bc_check_read() reports).
enum CheckSite : unsigned {
    CHECK_BC7_STAGE = 1,
    CHECK_BC7_SCRATCH = 2,
    CHECK_BC7_STORE = 3,
    CHECK_BC6H_STAGE = 4,
    CHECK_BC6H_SCRATCH = 5,
    CHECK_BC6H_STORE = 6,
    CHECK_BC15_LOAD = 7,
    CHECK_BC15_STORE = 8,
    CHECK_DECODE_SMEM = 9,
    CHECK_DECODE_STORE = 10,
    CHECK_SELFTEST = 11,
};

#ifdef BCN_CHECK
// This translation unit's record: site + 1 (0 = no failure), index, extent.
static __device__ unsigned long long g_check_rec[3];

__device__ __forceinline__ bool check_in_bounds(unsigned long long i, unsigned long long n, unsigned site) {
    if (i < n) return true;
    if (atomicCAS(&g_check_rec[0], 0ull, (unsigned long long)site + 1ull) == 0ull) {
        g_check_rec[1] = i;
        g_check_rec[2] = n;
    }
    return false;
}
#define BCN_GUARD(i, n, site) ::bcn::check_in_bounds((unsigned long long)(i), (unsigned long long)(n), (site))

// Host: copies this translation unit's record to out[3] and clears it.
static inline cudaError_t check_record_take(unsigned long long out[3]) {
    cudaError_t e = cudaMemcpyFromSymbol(out, g_check_rec, sizeof(unsigned long long) * 3);
    if (e != cudaSuccess) return e;
    const unsigned long long zero[3] = {0, 0, 0};
    return cudaMemcpyToSymbol(g_check_rec, zero, sizeof(zero));
}
#else
#define BCN_GUARD(i, n, site) true
static inline cudaError_t check_record_take(unsigned long long out[3]) {
    out[0] = out[1] = out[2] = 0;
    return cudaSuccess;
}
#endif

}  // namespace bcn
