// BC7 encoder for sm_100a.
//
// Work decomposition. Blocks are processed in tiles of 32 consecutive 4x4
// blocks; lane l of a warp always works on block l of its tile, so the 32
// lanes of a warp run the same mode and candidate (no intra-warp divergence
// apart from the per-block partition lists). The reference's per-block
// search (src/encode/bc7.rs:540-879) becomes a pipeline of launches, each
// running one narrow code path (a single fused kernel thrashed the
// instruction cache: every warp of an SM ran a different mode):
//
//   prep     PCA split bounds of the 64 partitions, ascending top-k lists
//            (modes 1/3/7)
//   search   modes 1/3/7 (modes 1 and 3 in one launch); grid (tile,
//            candidate group), a warp evaluates one partition candidate for
//            32 blocks; the first minimum per block is kept with a 64-bit
//            atomicMin on (error bits << 32 | candidate). Modes 0/2 (three
//            subsets, fixed partition order): one CTA per tile evaluates
//            each distinct subset of the searched partitions once and sums
//            them per partition
//   refine   one launch per mode: refinement of each block's winner + coding
//   mode4/5  rotation / index-swap candidates, one warp per candidate
//   mode6    one warp per tile
//   select   the reference's sequential "strictly better" scan over the
//            per-mode results -> one 128-bit store per block
//
// mode4/5 + mode6, search/refine of modes 0/2, and prep -> search/refine of
// modes 1/3/7 are independent chains, run on their own streams (the refines
// of modes 1/3/7 on a fourth one).
//
// Blocks are staged in shared memory as planar f32 with 128-bit coalesced
// loads. Every per-candidate computation keeps the reference's operation
// order, so the chosen mode, endpoints and indices are bit-identical to the
// reference CPU encoder (see bc_common.cuh for the float rules).
#include <cuda_runtime.h>

#include <climits>
#include <cstring>

#include "bc_common.cuh"
#include "bc_kernels.h"
#include "bptc_math.cuh"
#include "bc7_device.cuh"
#include "bc_check.cuh"

// Minimum resident CTAs per SM requested from the register allocator.
#ifndef BCN_MODE45_MINB
#define BCN_MODE45_MINB 7
#endif
#ifndef BCN_REFINE_MINB
#define BCN_REFINE_MINB 4
#endif
#ifndef BCN_REFINE_WARPS  // warps (tiles) per CTA of the refine and mode-6 kernels
#define BCN_REFINE_WARPS 4
#endif
static_assert(BCN_REFINE_WARPS >= 1 && BCN_REFINE_WARPS <= 4, "10.5 KiB of static shared memory per warp, 48 KiB at most");
#ifndef BCN_MODE6_MINB
#define BCN_MODE6_MINB 4
#endif
#ifndef BCN_PREP_MINB
#define BCN_PREP_MINB 4
#endif
#ifndef BCN_SEARCH_MINB  // search of modes 0-3
#define BCN_SEARCH_MINB 6
#endif
#ifndef BCN_SEARCH7_MINB  // mode 7 (4 channels) needs more registers
#define BCN_SEARCH7_MINB 5
#endif
#ifndef BCN_SEARCH3_WARPS  // warps per CTA of the mode 0/2 search (36 and 140 distinct subsets)
#define BCN_SEARCH3_WARPS 12
#endif
#ifndef BCN_SEARCH3_MINB
#define BCN_SEARCH3_MINB 4
#endif
namespace bcn {
namespace bc7 {

using namespace bptc;

// ---- kernels --------------------------------------------------------------------

// Candidate-mode index mi: 0 mode0, 1 mode2, 2 mode1, 3 mode3, 4 mode7 (the
// reference evaluation order, bc7.rs:853-867). Slots: mi for modes 0/2/1/3/7,
// then the mode-4 candidates, the mode-5 candidates, and mode 6.
struct Plan {
    int count[5];
    int k_a, k_b;        // top-k lengths of the two bound lists
    bool bounds_a, bounds_b;
    int n45_4, n45_5;    // mode-4 / mode-5 candidate counts
    bool run6;
};

static __host__ __device__ Plan make_plan(const BC7SettingsDev& s) {
    Plan p;
    bool ms0 = s.mode_selection[0] != 0, ms1 = s.mode_selection[1] != 0;
    bool run13 = ms1 && (s.fast_skip_threshold_mode1 != 0 || s.fast_skip_threshold_mode3 != 0);
    bool run7 = ms1 && s.fast_skip_threshold_mode7 != 0;
    p.count[0] = ms0 ? 16 : 0;
    p.count[1] = (ms0 && s.skip_mode2 == 0) ? 64 : 0;
    p.count[2] = run13 ? (int)s.fast_skip_threshold_mode1 : 0;
    p.count[3] = run13 ? (int)s.fast_skip_threshold_mode3 : 0;
    p.count[4] = run7 ? (int)s.fast_skip_threshold_mode7 : 0;
    // Mode 7's bounds use the settings' channel count; with 3 channels they
    // equal the mode 1/3 bounds and one sorted list serves both.
    bool sep7 = run7 && s.channels == 4;
    int t1 = (int)s.fast_skip_threshold_mode1, t3 = (int)s.fast_skip_threshold_mode3;
    int k13 = run13 ? (t1 > t3 ? t1 : t3) : 0;
    p.bounds_a = run13 || (run7 && !sep7);
    p.bounds_b = sep7;
    int k7 = (run7 && !sep7) ? (int)s.fast_skip_threshold_mode7 : 0;
    p.k_a = k13 > k7 ? k13 : k7;
    p.k_b = sep7 ? (int)s.fast_skip_threshold_mode7 : 0;
    int nrot = s.mode_selection[2] != 0 ? (int)s.channels - (int)s.mode45_channel0 : 0;
    if (nrot < 0) nrot = 0;
    p.n45_4 = 2 * nrot;
    p.n45_5 = nrot;
    p.run6 = s.mode_selection[3] != 0;
    return p;
}

// Arguments shared by every kernel of one encode. Scratch arrays are indexed
// [row * npad + tile * 32 + lane] so a warp's 32 lanes touch 32 consecutive
// entries. A single-image encode describes its image inline; a batched
// encode (tasks != nullptr) maps every global tile to the task it belongs to.
struct Work {
    const uint8_t* src;
    size_t stride;
    uint32_t bw, nblocks, npad;
    bool aligned;
    uint8_t* dst;
    const TaskDesc* tasks;     // batched encodes only
    const uint32_t* tile_task; // batched encodes only: task index of each tile
    uint8_t* lists;            // [row * npad + block]: rows 0..k_a-1 list A, then k_b rows of list B
    unsigned long long* keys;  // [mi * npad + block]: (error bits << 32) | candidate
    float* slot_err;           // [slot * npad + block]
    uint4* slot_data;          // [slot * npad + block]
    BC7SettingsDev S;
};

// Where the tile's blocks come from and go to.
struct TileLoc {
    const uint8_t* src;
    size_t stride;
    uint8_t* dst;
    uint32_t bw;
    uint32_t first;    // block index (within its image) of the tile's lane 0
    uint32_t nblocks;  // blocks of its image
    bool aligned;
    BCN_DEV bool valid(int lane) const { return first + lane < nblocks; }
};

BCN_DEV TileLoc tile_loc(const Work& w, uint32_t tile) {
    TileLoc t;
    if (w.tasks == nullptr) {
        t.src = w.src;
        t.stride = w.stride;
        t.dst = w.dst;
        t.bw = w.bw;
        t.first = tile * NB;
        t.nblocks = w.nblocks;
        t.aligned = w.aligned;
    } else {
        const TaskDesc& d = w.tasks[w.tile_task[tile]];
        t.src = d.src;
        t.stride = d.stride;
        t.dst = d.dst;
        t.bw = d.bw;
        t.first = (tile - d.tile_base) * NB;
        t.nblocks = d.bw * d.bh;
        t.aligned = d.aligned != 0;
    }
    return t;
}

// Row `row` of a scratch array with `rows` rows, at block gi: whether the
// guarded index is inside the array (always true outside check builds).
BCN_DEV bool scratch_ok(const Work& w, int row, int rows, uint32_t gi) {
    return BCN_GUARD(row, rows, CHECK_BC7_SCRATCH) && BCN_GUARD(gi, w.npad, CHECK_BC7_SCRATCH);
}
BCN_DEV int nslots_of(const Plan& P) { return 5 + P.n45_4 + P.n45_5 + 1; }

// Stages the 32 blocks of `tile` into px (planar f32, lane-strided) with
// threads tid = 0..nt-1 (128-bit loads: the 4 rows of 32 neighbouring blocks
// are 4 contiguous 512-byte spans). PK: also rows PX_PACKED.. (the pixel
// words as loaded), for the integer index fit.
template <bool PK = true>
BCN_DEV void stage_tile(float (*px)[NB], const Work& w, uint32_t tile, int tid, int nt) {
    const TileLoc L = tile_loc(w, tile);
    for (int t = tid; t < NB * 4; t += nt) {
        int b = t & 31, y = t >> 5;
        uint32_t gi = L.first + b;
        uint32_t v[4] = {0, 0, 0, 0};
        if (gi < L.nblocks) {
            uint32_t by = gi / L.bw, bx = gi - by * L.bw;
            // the image's rows and block columns
            if (!BCN_GUARD(by * 4 + y, (L.nblocks + L.bw - 1) / L.bw * 4, CHECK_BC7_STAGE) ||
                !BCN_GUARD(bx, L.bw, CHECK_BC7_STAGE))
                continue;
            const uint8_t* row = L.src + (size_t)(by * 4 + y) * L.stride + (size_t)bx * 16;
            if (L.aligned) {
                uint4 q = __ldg(reinterpret_cast<const uint4*>(row));
                v[0] = q.x;
                v[1] = q.y;
                v[2] = q.z;
                v[3] = q.w;
            } else {
                for (int j = 0; j < 16; j++) v[j >> 2] |= (uint32_t)row[j] << (8 * (j & 3));
            }
        }
#pragma unroll
        for (int x = 0; x < 4; x++) {
            int k = y * 4 + x;
            px[k][b] = (float)(v[x] & 0xFF);
            px[16 + k][b] = (float)((v[x] >> 8) & 0xFF);
            px[32 + k][b] = (float)((v[x] >> 16) & 0xFF);
            px[48 + k][b] = (float)(v[x] >> 24);
            if (PK) px[PX_PACKED + k][b] = __uint_as_float(v[x]);
        }
    }
}

// Rows PX_SQ..PX_SQ+3 of a staged tile: per block and channel, the sum of
// the squares of its 16 values (exact integers, below 2^24), stored as int
// bits. Threads tid = 0..nt-1, after the staged rows are visible to them.
BCN_DEV void stage_channel_squares(float (*px)[NB], int tid, int nt) {
    for (int t = tid; t < 4 * NB; t += nt) {
        const int c = t >> 5, b = t & 31;
        float s = 0.0f;
#pragma unroll
        for (int k = 0; k < 16; k++) s = fmaf(px[c * 16 + k][b], px[c * 16 + k][b], s);
        px[PX_SQ + c][b] = __int_as_float((int)s);
    }
}

template <class B>
BCN_DEV float opaque_err(const B& blk, uint32_t channels) {
    // compute_opaque_err (bc7.rs:869-879)
    float e = 0.0f;
    if (channels != 3)
        for (int k = 0; k < 16; k++) e += sqf(blk(3, k) - 255.0f);
    return e;
}

// The smaller subset (pixel mask) of a two-subset partition. A partition's
// bound is the sum of its two subsets' bounds, computed from one subset's
// statistics and the whole block's minus them (exact integers either way);
// the sum is the same whichever subset comes first (float addition is
// commutative), so the loop over pixels runs over the smaller subset: 6.4
// pixels on average over the 64 partitions instead of 8.7 for subset 0.
BCN_DEV uint32_t smaller_subset(uint32_t pattern) {
    const uint32_t m0 = subset_mask_from_map(pattern, 0);
    return __popc(m0) <= 8 ? m0 : ~m0 & 0xFFFFu;
}

// K1: PCA split bounds + ascending top-k partition lists (bc7.rs:622-655,
// 819-851; common.rs:126-140).
template <int NW>
__global__ void __launch_bounds__(NW * 32, BCN_PREP_MINB) bc7_prep_kernel(Work w) {
    __shared__ float px[64][NB];
    __shared__ int keys[2][64][NB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x, gi = tile * NB + lane;
    const Plan P = make_plan(w.S);
    stage_tile<false>(px, w, tile, threadIdx.x, NW * 32);
    __syncthreads();
    const Blk blk{&px[0][lane]};
    if (P.bounds_a && P.bounds_b) {
        // Both lists: the 4-channel statistics and covariance hold the
        // 3-channel ones (entries 0-2, 4, 5, 7, 10-12, 14 are the same sums
        // in the same order), so one pass per partition feeds both bounds.
        float full[15];
        stats_masked<4, true>(blk, 0xFFFFu, full);
        for (int part = warp; part < 64; part += NW) {
            float st[15], cv[10];
            stats_masked<4, true>(blk, smaller_subset(kPartitionMap[part]), st);
            covar_from_stats<4, true>(cv, st);
            float ba = 0.0f, bb = 0.0f;
            ba += pca_bound<3>(cv);
            bb += pca_bound<4>(cv);
#pragma unroll
            for (int i = 0; i < 15; i++) st[i] = full[i] - st[i];
            covar_from_stats<4, true>(cv, st);
            ba += pca_bound<3>(cv);
            bb += pca_bound<4>(cv);
            keys[0][part][lane] = part + (int)(sqrtf(ba) * 256.0f) * 64;
            keys[1][part][lane] = part + (int)(sqrtf(bb) * 256.0f) * 64;
        }
    } else if (P.bounds_a || P.bounds_b) {
        const int set = P.bounds_a ? 0 : 1;
        float full[15];
        if (set == 0) stats_masked<3, true>(blk, 0xFFFFu, full);
        else stats_masked<4, true>(blk, 0xFFFFu, full);
        for (int part = warp; part < 64; part += NW) {
            uint32_t mask = smaller_subset(kPartitionMap[part]);
            float b12 = set == 0 ? pca_bound_split<3, true>(blk, mask, full) : pca_bound_split<4, true>(blk, mask, full);
            keys[set][part][lane] = part + (int)b12 * 64;
        }
    }
    __syncthreads();
    // partial_sort_list: keys are unique, so the first K entries are the K
    // smallest in ascending order. Tournament selection: the minima of 8
    // groups of 8 keys; each step takes the smallest group minimum (the low
    // 6 bits of a key are its partition, so also its group) and rescans only
    // that group.
    for (int set = 0; set < 2; set++) {
        int K = set == 0 ? P.k_a : P.k_b;
        if (K == 0 || warp != set) continue;
        int gm[8];
#pragma unroll
        for (int g = 0; g < 8; g++) {
            int m = INT_MAX;
#pragma unroll
            for (int i = 0; i < 8; i++) m = min(m, keys[set][8 * g + i][lane]);
            gm[g] = m;
        }
        for (int k = 0; k < K; k++) {
            int best = gm[0];
#pragma unroll
            for (int g = 1; g < 8; g++) best = min(best, gm[g]);
            const int bi = best & 63, bg = bi >> 3;
            keys[set][bi][lane] = INT_MAX;
            int m = INT_MAX;
#pragma unroll
            for (int i = 0; i < 8; i++) m = min(m, keys[set][8 * bg + i][lane]);
#pragma unroll
            for (int g = 0; g < 8; g++) gm[g] = g == bg ? m : gm[g];
            const int row = set == 0 ? k : P.k_a + k;
            if (scratch_ok(w, row, P.k_a + P.k_b, gi)) w.lists[(size_t)row * w.npad + gi] = (uint8_t)bi;
        }
    }
}

BCN_DEV int part_of(const Work& w, int mi, int c, uint32_t gi, const Plan& P) {
    if (mi <= 1) return c + 64;  // modes 0 and 2: partitions 0..count-1 of the 3-subset table
    int row = (mi == 4 && P.bounds_b) ? P.k_a + c : c;
    return scratch_ok(w, row, P.k_a + P.k_b, gi) ? w.lists[(size_t)row * w.npad + gi] : 0;
}

// K2: every partition candidate of modes 1, 3 and 7 (bc7.rs:517-569). Grid:
// (tile, candidate group); warp w evaluates candidate blockIdx.y*NW+w for
// the 32 blocks of the tile. The CTA's first minimum per block goes to the
// global argmin key with a 64-bit atomicMin -- errors are non-negative, so
// their bit patterns order like the values, and the low word breaks ties
// toward the earlier candidate, exactly the reference's strict "<" scan.
// MODE 13 runs modes 1 and 3 together: both take their candidates from the
// same sorted partition list, so candidate c is the same partition in both,
// and its unquantised endpoints (segment_part2) are computed once for the
// two.
template <int MODE, int NW>
__global__ void __launch_bounds__(NW * 32, (MODE == 7 ? BCN_SEARCH7_MINB : BCN_SEARCH_MINB) * 8 / NW)
    bc7_search_kernel(Work w) {
    static_assert(MODE == 1 || MODE == 3 || MODE == 7 || MODE == 13, "two-subset modes");
    constexpr int CH = MODE == 7 ? 4 : 3;
    constexpr int mia = MODE == 3 ? 3 : (MODE == 7 ? 4 : 2);  // candidate-mode index (mode 1 for 13)
    constexpr int NK = MODE == 13 ? 2 : 1;
    __shared__ float px[PX_ROWS][NB];
    __shared__ float full[15][NB];
    __shared__ unsigned long long best[NK][NW][NB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x, gi = tile * NB + lane;
    const Plan P = make_plan(w.S);
    stage_tile(px, w, tile, threadIdx.x, NW * 32);
    __syncthreads();
    const Blk blk{&px[0][lane]};
    // the whole block's statistics, one entry per warp at a time, and the
    // channel square sums
    for (int e = warp; e < 15; e += NW) full[e][lane] = stat_entry<CH>(blk, e);
    stage_channel_squares(px, threadIdx.x, NW * 32);
    __syncthreads();
    const int c = blockIdx.y * NW + warp;
    const int na = P.count[mia], nb = MODE == 13 ? P.count[3] : 0;
    unsigned long long key[NK];
#pragma unroll
    for (int i = 0; i < NK; i++) key[i] = ~0ull;
    auto key_of = [&](float err) {
        return err == err ? ((unsigned long long)__float_as_uint(err) << 32) | (uint32_t)c : ~0ull;
    };
    if (c < max(na, nb) && tile_loc(w, tile).valid(lane)) {
        const uint32_t pattern = kPartitionMap[part_of(w, mia, c, gi, P)];
        float ep[16];
        segment_part2<CH>(blk, pattern, &full[0][lane], ep);
        if (MODE == 13) {
            if (c < nb) {
                float e3[16];
#pragma unroll
                for (int i = 0; i < 16; i++) e3[i] = ep[i];
                key[NK - 1] = key_of(quant_fit_part2<3>(blk, pattern, e3));
            }
            if (c < na) key[0] = key_of(quant_fit_part2<1>(blk, pattern, ep));
        } else {
            key[0] = key_of(quant_fit_part2<MODE>(blk, pattern, ep));
        }
    }
#pragma unroll
    for (int i = 0; i < NK; i++) best[i][warp][lane] = key[i];
    __syncthreads();
    if (warp < NK) {
        const int mi = warp == 0 ? mia : 3;
        unsigned long long k = best[warp][0][lane];
        for (int i = 1; i < NW; i++) k = min(k, best[warp][i][lane]);
        if (k != ~0ull && scratch_ok(w, mi, 5, gi)) atomicMin(&w.keys[(size_t)mi * w.npad + gi], k);
    }
}

// The distinct pixel subsets of the first NPART three-subset partitions
// (modes 0 and 2 search partitions 0..15 and 0..63 of that table), in order
// of first appearance, and each partition's three subsets as indices into
// that list: 36 distinct subsets among the 48 of mode 0, 140 among the 192
// of mode 2.
constexpr uint32_t kPartitionMapHost[128] = {BCN_PARTITION_MAP_VALUES};

template <int NPART>
struct Subsets3 {
    static constexpr int kMax = 3 * NPART;
    uint16_t mask[kMax];
    uint8_t idx[NPART][3];
    int count;
};

template <int NPART>
constexpr Subsets3<NPART> make_subsets3() {
    Subsets3<NPART> t{};
    t.count = 0;
    for (int p = 0; p < NPART; p++) {
        for (int j = 0; j < 3; j++) {
            uint32_t m = 0;
            for (int k = 0; k < 16; k++)
                if (((kPartitionMapHost[64 + p] >> (2 * k)) & 3u) == (uint32_t)j) m |= 1u << k;
            int u = 0;
            while (u < t.count && t.mask[u] != m) u++;
            if (u == t.count) t.mask[t.count++] = (uint16_t)m;
            t.idx[p][j] = (uint8_t)u;
        }
    }
    return t;
}

constexpr Subsets3<16> kSubsets0Host = make_subsets3<16>();
constexpr Subsets3<64> kSubsets2Host = make_subsets3<64>();
static_assert(kSubsets0Host.count == 36 && kSubsets2Host.count == 140, "distinct subsets of modes 0 / 2");
__constant__ Subsets3<16> kSubsets0 = make_subsets3<16>();
__constant__ Subsets3<64> kSubsets2 = make_subsets3<64>();

// Which warp of a CTA of NW evaluates which distinct subset: longest first,
// each to the warp with the least work so far, at an estimated cost of
// 300 + 70 * (pixels) instructions per subset (a fixed endpoint fit plus
// per-pixel statistics, projection and index fit). Subsets of 1 to 14
// pixels differ in cost by about 3x, and the CTA waits for its slowest warp
// before the partition sums. order[start[w] .. start[w + 1]) are warp w's
// subsets.
template <int NPART, int NW>
struct SubsetSchedule {
    uint8_t order[3 * NPART];
    uint8_t start[NW + 1];
};

template <int NPART, int NW>
constexpr SubsetSchedule<NPART, NW> make_schedule(const Subsets3<NPART>& t) {
    SubsetSchedule<NPART, NW> r{};
    int owner[3 * NPART] = {};
    bool done[3 * NPART] = {};
    int load[NW] = {};
    for (int n = 0; n < t.count; n++) {
        int best = -1, bc = -1;
        for (int u = 0; u < t.count; u++) {
            int pc = 0;
            for (uint32_t m = t.mask[u]; m; m &= m - 1) pc++;
            if (!done[u] && 300 + 70 * pc > bc) {
                bc = 300 + 70 * pc;
                best = u;
            }
        }
        int w = 0;
        for (int i = 1; i < NW; i++)
            if (load[i] < load[w]) w = i;
        done[best] = true;
        owner[best] = w;
        load[w] += bc;
    }
    int pos = 0;
    for (int w = 0; w < NW; w++) {
        r.start[w] = (uint8_t)pos;
        for (int u = 0; u < t.count; u++)
            if (owner[u] == w) r.order[pos++] = (uint8_t)u;
    }
    r.start[NW] = (uint8_t)pos;
    return r;
}

__constant__ SubsetSchedule<16, BCN_SEARCH3_WARPS> kSchedule0 = make_schedule<16, BCN_SEARCH3_WARPS>(kSubsets0Host);
__constant__ SubsetSchedule<64, BCN_SEARCH3_WARPS> kSchedule2 = make_schedule<64, BCN_SEARCH3_WARPS>(kSubsets2Host);

// K2 for modes 0 and 2 (bc7.rs:517-569 over partitions 0..count-1 in table
// order). One CTA per tile: the warps evaluate the mode's distinct subsets
// (eval_subset, one subset for the tile's 32 blocks per warp at a time, in
// the order of the subset schedule),
// then each partition's error is the sum of its three subsets' errors plus
// the block's v . v -- exact integers below 2^24, so the same float as the
// reference's pixel-order sum -- and the first minimum over the partitions
// goes to the argmin key.
template <int MODE, int NW>
__global__ void __launch_bounds__(NW * 32, BCN_SEARCH3_MINB) bc7_search3_kernel(Work w) {
    constexpr int mi = MODE == 0 ? 0 : 1;
    constexpr int NPART = MODE == 0 ? 16 : 64, NS = MODE == 0 ? 36 : 140;
    const Subsets3<NPART>& T = *(MODE == 0 ? (const Subsets3<NPART>*)&kSubsets0 : (const Subsets3<NPART>*)&kSubsets2);
    __shared__ float px[PX_ROWS][NB];
    __shared__ int serr[NS][NB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x, gi = tile * NB + lane;
    const Plan P = make_plan(w.S);
    stage_tile(px, w, tile, threadIdx.x, NW * 32);
    __syncthreads();
    stage_channel_squares(px, threadIdx.x, NW * 32);
    __syncthreads();
    const Blk blk{&px[0][lane]};
    const int count = min(P.count[mi], NPART);
    const bool valid = tile_loc(w, tile).valid(lane);
    static_assert(NW == BCN_SEARCH3_WARPS, "the subset schedules are made for BCN_SEARCH3_WARPS warps");
    const SubsetSchedule<NPART, NW>& S =
        *(MODE == 0 ? (const SubsetSchedule<NPART, NW>*)&kSchedule0 : (const SubsetSchedule<NPART, NW>*)&kSchedule2);
    for (int i = S.start[warp]; i < S.start[warp + 1]; i++) {
        const int u = S.order[i];
        serr[u][lane] = valid ? eval_subset<MODE>(blk, T.mask[u]) : 0;
    }
    __syncthreads();
    if (warp != 0 || !valid || count == 0) return;
    const int v2 = block_sq<3>(blk);
    unsigned long long key = ~0ull;
    for (int c = 0; c < count; c++) {
        const int total = serr[T.idx[c][0]][lane] + serr[T.idx[c][1]][lane] + serr[T.idx[c][2]][lane] + v2;
        key = min(key, ((unsigned long long)__float_as_uint((float)total) << 32) | (uint32_t)c);
    }
    if (scratch_ok(w, mi, 5, gi)) atomicMin(&w.keys[(size_t)mi * w.npad + gi], key);
}

// K3: refinement of each block's winning partition + coding (bc7.rs:571-609).
// One warp per tile.
template <int MODE, int NW>
__global__ void __launch_bounds__(NW * 32, BCN_REFINE_MINB) bc7_refine_kernel(Work w, uint32_t ntiles) {
    constexpr int mi = MODE == 0 ? 0 : (MODE == 2 ? 1 : (MODE == 1 ? 2 : (MODE == 3 ? 3 : 4)));
    __shared__ float px[NW][PX_ROWS][NB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x * NW + warp;
    if (tile >= ntiles) return;
    stage_tile(px[warp], w, tile, lane, 32);
    __syncwarp();
    stage_channel_squares(px[warp], lane, 32);
    __syncwarp();
    const uint32_t gi = tile * NB + lane;
    const Plan P = make_plan(w.S);
    const Blk blk{&px[warp][0][lane]};
    unsigned long long key = scratch_ok(w, mi, 5, gi) ? w.keys[(size_t)mi * w.npad + gi] : ~0ull;
    float err = __int_as_float(0x7f800000);
    uint4 data = make_uint4(0, 0, 0, 0);
    if (key != ~0ull && tile_loc(w, tile).valid(lane)) {
        int c = (int)(key & 0xFFFFFFFFu);
        float e0 = __uint_as_float((uint32_t)(key >> 32));
        int iters = (int)w.S.refine_iterations[MODE];
        err = refine_and_code<MODE>(blk, kPartitionMap, part_of(w, mi, c, gi, P), e0, iters,
                                    opaque_err(blk, w.S.channels), data);
    }
    if (scratch_ok(w, mi, nslots_of(P), gi)) {
        w.slot_err[(size_t)mi * w.npad + gi] = err;
        w.slot_data[(size_t)mi * w.npad + gi] = data;
    }
}

// K4: mode 4 / mode 5 rotation candidates (bc7.rs:657-760); mode 4 runs one
// launch per index-swap setting. Grid: (tile, rotation group), warp = one
// rotation for the tile's 32 blocks.
template <int MODE, int SWAP, bool CH4, int NW>
__global__ void __launch_bounds__(NW * 32, BCN_MODE45_MINB) bc7_mode45_kernel(Work w) {
    __shared__ float px[PX_ROWS][NB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x, gi = tile * NB + lane;
    const Plan P = make_plan(w.S);
    stage_tile(px, w, tile, threadIdx.x, NW * 32);
    if (!CH4) {
        // 3-channel settings: the rotated-out channel reads 255 (BlkRot)
        __syncthreads();
        for (int t = threadIdx.x; t < 16 * NB; t += NW * 32) {
            px[48 + t / NB][t % NB] = 255.0f;
            px[PX_PACKED + t / NB][t % NB] =
                __uint_as_float(__float_as_uint(px[PX_PACKED + t / NB][t % NB]) | 0xFF000000u);
        }
    }
    __syncthreads();
    stage_channel_squares(px, threadIdx.x, NW * 32);
    __syncthreads();
    const int r = blockIdx.y * NW + warp;  // rotation index
    if (r >= P.n45_5) return;              // n45_5 = number of rotations
    int rot = (int)w.S.mode45_channel0 + r;
    uint4 data;
    float err = mode45_candidate<MODE, SWAP, CH4>(&px[0][lane], w.S.refine_iterations[MODE],
                                                  w.S.refine_iterations_channel, rot, data);
    // candidate order of the reference: mode 4 (rotation, swap 0), (rotation,
    // swap 1), ... then mode 5 rotations
    int slot = 5 + (MODE == 4 ? 2 * r + SWAP : P.n45_4 + r);
    if (scratch_ok(w, slot, nslots_of(P), gi)) {
        w.slot_err[(size_t)slot * w.npad + gi] = err;
        w.slot_data[(size_t)slot * w.npad + gi] = data;
    }
}

// K5: mode 6 (bc7.rs:762-817), one warp per tile.
template <int CH, int NW>
__global__ void __launch_bounds__(NW * 32, BCN_MODE6_MINB) bc7_mode6_kernel(Work w, uint32_t ntiles) {
    __shared__ float px[NW][PX_ROWS][NB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x * NW + warp;
    if (tile >= ntiles) return;
    stage_tile(px[warp], w, tile, lane, 32);
    __syncwarp();
    stage_channel_squares(px[warp], lane, 32);
    __syncwarp();
    const Plan P = make_plan(w.S);
    const uint32_t gi = tile * NB + lane;
    const Blk blk{&px[warp][0][lane]};
    uint4 data;
    float err = mode6<CH>(blk, w.S.refine_iterations[6], data);
    int slot = 5 + P.n45_4 + P.n45_5;
    if (scratch_ok(w, slot, nslots_of(P), gi)) {
        w.slot_err[(size_t)slot * w.npad + gi] = err;
        w.slot_data[(size_t)slot * w.npad + gi] = data;
    }
}

// K6: the reference keeps a candidate only when its error is strictly below
// the best so far, scanning modes 0,2,1,3,7, the mode-4 then mode-5
// candidates, then mode 6 (bc7.rs:602-609, 735-760, 813-816): the first slot
// holding the minimum wins. A block no mode encodes stays all-zero.
__global__ void __launch_bounds__(256) bc7_select_kernel(Work w, uint32_t ntiles) {
    const uint32_t tile = blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (tile >= ntiles) return;
    const TileLoc L = tile_loc(w, tile);
    if (!L.valid(lane)) return;
    const uint32_t gi = tile * NB + lane;
    const Plan P = make_plan(w.S);
    float best = __int_as_float(0x7f800000);
    int win = -1;
    const int nslots = nslots_of(P);
    auto slot_err = [&](int s) {
        return scratch_ok(w, s, nslots, gi) ? w.slot_err[(size_t)s * w.npad + gi] : __int_as_float(0x7f800000);
    };
    for (int s = 0; s < 5; s++)
        if (P.count[s] > 0) {
            float e = slot_err(s);
            if (e < best) {
                best = e;
                win = s;
            }
        }
    const int n45 = P.n45_4 + P.n45_5;
    for (int s = 5; s < 5 + n45; s++) {
        float e = slot_err(s);
        if (e < best) {
            best = e;
            win = s;
        }
    }
    if (P.run6) {
        int s = 5 + n45;
        float e = slot_err(s);
        if (e < best) {
            best = e;
            win = s;
        }
    }
    uint4 data = win >= 0 && scratch_ok(w, win, nslots, gi) ? w.slot_data[(size_t)win * w.npad + gi]
                                                             : make_uint4(0, 0, 0, 0);
    if (!BCN_GUARD(L.first + lane, L.nblocks, CHECK_BC7_STORE)) return;
    uint8_t* o = L.dst + (size_t)(L.first + lane) * 16;
    if (((uintptr_t)L.dst & 15) == 0) {
        *reinterpret_cast<uint4*>(o) = data;
    } else {
        uint32_t* o32 = reinterpret_cast<uint32_t*>(o);
        o32[0] = data.x;
        o32[1] = data.y;
        o32[2] = data.z;
        o32[3] = data.w;
    }
}

}  // namespace bc7

cudaError_t check_take_bc7(unsigned long long out[3]) { return check_record_take(out); }

size_t bc7_scratch_bytes_tiles(uint32_t ntiles, const BC7SettingsDev& s) {
    const bc7::Plan P = bc7::make_plan(s);
    size_t npad = (size_t)ntiles * bc7::NB;
    int nslots = 5 + P.n45_4 + P.n45_5 + 1;
    return npad * ((size_t)(P.k_a + P.k_b) + 5 * 8 + (size_t)nslots * (4 + 16)) + 256;
}

size_t bc7_scratch_bytes(uint32_t nblocks, const BC7SettingsDev& s) {
    return bc7_scratch_bytes_tiles((nblocks + bc7::NB - 1) / bc7::NB, s);
}

namespace bc7 {

// Carves the scratch arrays out of `scratch` and enqueues the pipeline over
// `ntiles` tiles.
// The side streams of run_pipeline, with their fork, join and per-search
// events; per thread and device, created on first use.
struct SideStream {
    cudaStream_t st = nullptr, st2 = nullptr, st3 = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, join2 = nullptr, join3 = nullptr, searched[3] = {};
    int device = -1;
    void release() {
        for (cudaEvent_t* ev : {&fork, &join, &join2, &join3, &searched[0], &searched[1], &searched[2]})
            if (*ev) {
                cudaEventDestroy(*ev);
                *ev = nullptr;
            }
        for (cudaStream_t* q : {&st, &st2, &st3})
            if (*q) {
                cudaStreamDestroy(*q);
                *q = nullptr;
            }
        device = -1;
    }
    ~SideStream() { release(); }
    cudaError_t get() {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess || dev == device) return e;
        release();
        // non-blocking: no implicit ordering with the legacy default stream,
        // only the explicit fork / join events
        for (cudaStream_t* q : {&st, &st2, &st3})
            if ((e = cudaStreamCreateWithFlags(q, cudaStreamNonBlocking)) != cudaSuccess) return e;
        for (cudaEvent_t* ev : {&fork, &join, &join2, &join3, &searched[0], &searched[1], &searched[2]})
            if ((e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming)) != cudaSuccess) return e;
        device = dev;
        return cudaSuccess;
    }
};
static thread_local SideStream t_side;

static cudaError_t run_pipeline(Work& w, uint32_t ntiles, void* scratch, int search_warps, cudaStream_t s,
                                bool side_stream) {
    const Plan P = make_plan(w.S);
    size_t npad = (size_t)ntiles * NB;
    int nslots = 5 + P.n45_4 + P.n45_5 + 1;
    w.npad = (uint32_t)npad;
    uint8_t* p = (uint8_t*)(((uintptr_t)scratch + 255) & ~(uintptr_t)255);
    w.slot_data = (uint4*)p;
    p += npad * 16 * nslots;
    w.keys = (unsigned long long*)p;
    p += npad * 8 * 5;
    w.slot_err = (float*)p;
    p += npad * 4 * nslots;
    w.lists = p;

    constexpr int NWP = 8, NWR = BCN_REFINE_WARPS, NW45 = 4;
    auto groups = [](int count, int nw) { return (unsigned)((count + nw - 1) / nw); };
    unsigned rgrid = (ntiles + NWR - 1) / NWR;
    // argmin keys of the five searches: all ones = no candidate yet
    {
        cudaError_t e = cudaMemsetAsync(w.keys, 0xFF, npad * 8 * 5, s);
        if (e != cudaSuccess) return e;
    }
    // Three chains that only meet at the selection: mode 4/5 + mode 6 (read
    // only the tile), modes 0/2 (search + refine over the fixed partition
    // order) and prep -> modes 1/3/7. On their own streams (forked here,
    // joined before the selection) their launches overlap and fill the SMs
    // each launch's last wave leaves idle.
    cudaStream_t s2 = s, s3 = s;
    if (side_stream) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaError_t e = cudaStreamIsCapturing(s, &cs);
        if (e != cudaSuccess) return e;
        int dev = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        // while `s` captures a graph the side streams join the capture
        // through the fork event, but are not created then
        // (bc7_side_streams_init() makes them beforehand)
        if (cs == cudaStreamCaptureStatusNone || t_side.device == dev) {
            if ((e = t_side.get()) != cudaSuccess) return e;
            if ((e = cudaEventRecord(t_side.fork, s)) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(t_side.st, t_side.fork, 0)) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(t_side.st2, t_side.fork, 0)) != cudaSuccess) return e;
            s2 = t_side.st;
            s3 = t_side.st2;
        }
    }
    if (P.n45_5) {
        dim3 g45(ntiles, groups(P.n45_5, NW45));
        if (w.S.channels == 4) {
            bc7_mode45_kernel<4, 0, true, NW45><<<g45, NW45 * 32, 0, s2>>>(w);
            bc7_mode45_kernel<4, 1, true, NW45><<<g45, NW45 * 32, 0, s2>>>(w);
            bc7_mode45_kernel<5, 0, true, NW45><<<g45, NW45 * 32, 0, s2>>>(w);
        } else {
            bc7_mode45_kernel<4, 0, false, NW45><<<g45, NW45 * 32, 0, s2>>>(w);
            bc7_mode45_kernel<4, 1, false, NW45><<<g45, NW45 * 32, 0, s2>>>(w);
            bc7_mode45_kernel<5, 0, false, NW45><<<g45, NW45 * 32, 0, s2>>>(w);
        }
    }
    if (P.run6) {
        if (w.S.channels == 3) bc7_mode6_kernel<3, NWR><<<rgrid, NWR * 32, 0, s2>>>(w, ntiles);
        else bc7_mode6_kernel<4, NWR><<<rgrid, NWR * 32, 0, s2>>>(w, ntiles);
    }
    // K2 of modes 1/3/7; mode 13 = modes 1 and 3 in one launch
    auto search = [&](int mode, int count, cudaStream_t st) {
        // 4 candidates per CTA when 8 would leave a last group at most half
        // full (e.g. 12 candidates: 3 full CTAs of 4 instead of 8 + 4)
        const int rem = count % 8;
        if (search_warps == 4 || (rem != 0 && rem <= 4)) {
            dim3 g(ntiles, groups(count, 4));
            switch (mode) {
                case 13: bc7_search_kernel<13, 4><<<g, 128, 0, st>>>(w); break;
                case 1: bc7_search_kernel<1, 4><<<g, 128, 0, st>>>(w); break;
                case 3: bc7_search_kernel<3, 4><<<g, 128, 0, st>>>(w); break;
                default: bc7_search_kernel<7, 4><<<g, 128, 0, st>>>(w); break;
            }
        } else {
            dim3 g(ntiles, groups(count, 8));
            switch (mode) {
                case 13: bc7_search_kernel<13, 8><<<g, 256, 0, st>>>(w); break;
                case 1: bc7_search_kernel<1, 8><<<g, 256, 0, st>>>(w); break;
                case 3: bc7_search_kernel<3, 8><<<g, 256, 0, st>>>(w); break;
                default: bc7_search_kernel<7, 8><<<g, 256, 0, st>>>(w); break;
            }
        }
    };
    // modes 0 and 2 search partitions in table order: no prep needed
    constexpr int NW3 = BCN_SEARCH3_WARPS;
    if (P.count[0]) bc7_search3_kernel<0, NW3><<<ntiles, NW3 * 32, 0, s3>>>(w);
    if (P.count[1]) bc7_search3_kernel<2, NW3><<<ntiles, NW3 * 32, 0, s3>>>(w);
    if (P.count[0]) bc7_refine_kernel<0, NWR><<<rgrid, NWR * 32, 0, s3>>>(w, ntiles);
    if (P.count[1]) bc7_refine_kernel<2, NWR><<<rgrid, NWR * 32, 0, s3>>>(w, ntiles);
    bc7_prep_kernel<NWP><<<ntiles, NWP * 32, 0, s>>>(w);
    // modes 1/3/7: each refine starts on a fourth stream as soon as its own
    // search is done, overlapping the next searches (the refine kernels are
    // latency-bound at 16 warps per SM). Modes 1 and 3 search together.
    const bool split = s2 != s;
    auto after_search = [&](int ev) -> cudaError_t {
        if (!split) return cudaSuccess;
        cudaError_t e = cudaEventRecord(t_side.searched[ev], s);
        if (e != cudaSuccess) return e;
        return cudaStreamWaitEvent(t_side.st3, t_side.searched[ev], 0);
    };
    cudaStream_t sr = split ? t_side.st3 : s;
    if (P.count[2] || P.count[3]) {
        if (P.count[2] && P.count[3]) search(13, max(P.count[2], P.count[3]), s);
        else if (P.count[2]) search(1, P.count[2], s);
        else search(3, P.count[3], s);
        cudaError_t e = after_search(0);
        if (e != cudaSuccess) return e;
        if (P.count[2]) bc7_refine_kernel<1, NWR><<<rgrid, NWR * 32, 0, sr>>>(w, ntiles);
        if (P.count[3]) bc7_refine_kernel<3, NWR><<<rgrid, NWR * 32, 0, sr>>>(w, ntiles);
    }
    if (P.count[4]) {
        search(7, P.count[4], s);
        cudaError_t e = after_search(1);
        if (e != cudaSuccess) return e;
        bc7_refine_kernel<7, NWR><<<rgrid, NWR * 32, 0, sr>>>(w, ntiles);
    }
    if (split) {
        cudaError_t e = cudaEventRecord(t_side.join, s2);
        if (e != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s, t_side.join, 0)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(t_side.join2, s3)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s, t_side.join2, 0)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(t_side.join3, t_side.st3)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s, t_side.join3, 0)) != cudaSuccess) return e;
    }
    bc7_select_kernel<<<(ntiles + 7) / 8, 256, 0, s>>>(w, ntiles);
    return cudaGetLastError();
}

}  // namespace bc7

cudaError_t launch_bc7_encode(const uint8_t* src, size_t stride, uint32_t bw, uint32_t bh, uint8_t* dst,
                              const BC7SettingsDev& settings, void* scratch, cudaStream_t s, bool side_stream) {
    using namespace bc7;
    uint32_t n = bw * bh;
    if (n == 0) return cudaSuccess;
    Work w;
    w.src = src;
    w.stride = stride;
    w.bw = bw;
    w.nblocks = n;
    w.aligned = ((uintptr_t)src % 16 == 0) && (stride % 16 == 0);
    w.dst = dst;
    w.tasks = nullptr;
    w.tile_task = nullptr;
    w.S = settings;
    return run_pipeline(w, (n + NB - 1) / NB, scratch, 8, s, side_stream);
}

cudaError_t bc7_side_streams_init() { return bc7::t_side.get(); }

cudaError_t launch_bc7_batch(const TaskDesc* tasks_dev, const uint32_t* tile_task_dev, uint32_t ntiles,
                             const BC7SettingsDev& settings, void* scratch, int search_warps, cudaStream_t s) {
    using namespace bc7;
    if (ntiles == 0) return cudaSuccess;
    Work w;
    memset(&w, 0, sizeof(w));
    w.tasks = tasks_dev;
    w.tile_task = tile_task_dev;
    w.S = settings;
    return run_pipeline(w, ntiles, scratch, search_warps, s, true);
}

}  // namespace bcn

// ---- allocation-free BC7 entry point ---------------------------------------------
//
// bc_compress_bc7_device_noalloc runs the same kernels as the regular entry
// point, with their scratch in the fixed array below instead of memory
// allocated per call, for callers that may not allocate device memory during
// the call (see include/bc_capi.h).

#include <mutex>

#include "../../include/bc_capi.h"

namespace bcn {
namespace {

static __device__ __align__(256) uint8_t g_bc7_noalloc_scratch[BC_NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mu;
// Device address of the array per device ordinal, with the context it was
// looked up in: after a device reset the device gets a new primary context,
// the library's module is loaded again, and the address is looked up anew.
struct NoallocAddr {
    void* ctx;
    void* addr;
};
NoallocAddr g_noalloc_addr[64];

// The current context (the driver's cuCtxGetCurrent, reached through the
// runtime, so the library needs no link against the driver library).
typedef int (*CtxGetCurrentFn)(void**);
void* current_context() {
    static CtxGetCurrentFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return (CtxGetCurrentFn)f;
    }();
    void* ctx = nullptr;
    if (fn == nullptr || fn(&ctx) != 0) return nullptr;
    return ctx;
}

// Device address of the array on the current device. The array's name in host
// code is only a host-side handle; the kernels need the address the runtime
// reports for the current device, looked up once per device (and again
// after the device's context was replaced by a reset).
int noalloc_scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        record_cuda_error(e);
        return BC_ERR_CUDA;
    }
    if (dev < 0 || dev >= 64) return BC_ERR_NO_DEVICE;
    // make the device's primary context current on this thread (CUDA 12's
    // cudaSetDevice initialises it), so the context read below is the one
    // the launches use
    e = cudaSetDevice(dev);
    if (e != cudaSuccess) {
        record_cuda_error(e);
        return BC_ERR_CUDA;
    }
    void* ctx = current_context();
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev].addr || ctx == nullptr || g_noalloc_addr[dev].ctx != ctx) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_bc7_noalloc_scratch);
        if (e != cudaSuccess) {
            record_cuda_error(e);
            return BC_ERR_CUDA;
        }
        g_noalloc_addr[dev].addr = p;
        g_noalloc_addr[dev].ctx = ctx;
    }
    *out = g_noalloc_addr[dev].addr;
    return BC_OK;
}

}  // namespace
}  // namespace bcn

extern "C" int bc_compress_bc7_device_noalloc(const bc_bc7_settings* settings, const uint8_t* rgba_dev,
                                              size_t rgba_len, uint8_t* blocks_dev, size_t blocks_len,
                                              uint32_t width, uint32_t height, size_t stride_bytes, void* stream) {
    using namespace bcn;
    // The checks of bc_compress_rgba8_device (src/encode.rs:91-101).
    if (height % 4 != 0 || width % 4 != 0) return BC_ERR_DIMS;
    int rc = validate_bc7_settings(settings);
    if (rc != BC_OK) return rc;
    uint32_t bw = width / 4, bh = height / 4;
    if (blocks_len < (size_t)bw * bh * 16) return BC_ERR_DST_SIZE;
    if (width > 0 && height > 0 && rgba_len < (size_t)(height - 1) * stride_bytes + (size_t)width * 4)
        return BC_ERR_SRC_SIZE;
    if (width == 0 || height == 0) return BC_OK;
    if (!rgba_dev || !blocks_dev) return BC_ERR_NULL;
    const BC7SettingsDev& s7 = *reinterpret_cast<const BC7SettingsDev*>(settings);
    if (bc7_scratch_bytes(bw * bh, s7) > BC_NOALLOC_SCRATCH_BYTES) return BC_ERR_TOO_LARGE;
    void* scratch = nullptr;
    rc = noalloc_scratch_address(&scratch);
    if (rc != BC_OK) return rc;
    // single stream: this entry point creates no resources
    cudaError_t e =
        launch_bc7_encode(rgba_dev, stride_bytes, bw, bh, blocks_dev, s7, scratch, (cudaStream_t)stream, false);
    if (e != cudaSuccess) {
        record_cuda_error(e);
        return BC_ERR_CUDA;
    }
    return BC_OK;
}
