// Batched compression: every pending task of a bc_compressor -- many
// textures, mip levels and variants -- frozen into one device task table and
// replayed as one CUDA graph.
//
//   BC1-BC5 tasks  one persistent work-queue launch over all their tiles
//   BC7 tasks      one pass of the BC7 pipeline over all tiles of all tasks
//                  that share settings (each phase is a single launch)
//   BC6H tasks     one pass of the BC6H kernel pipeline per task
//
// The launch shape (threads per CTA, resident CTAs per SM, tiles per
// work-queue claim, candidates per BC7 search CTA) comes from a bc_tune
// value, which bc_batch_create can pick by timing the candidates on the
// batch itself (autotune); chosen values are cached per device and batch
// shape for the life of the process.
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/bc_capi.h"
#include "bc_kernels.h"

namespace bcn {

// The task record bc_compressor keeps (capi.cu).
struct BcTaskView {
    int variant;
    const void* settings;
    const uint8_t* src;
    size_t pitch;
    uint32_t w, h;
    uint8_t* dst;
};
int compressor_tasks(bc_compressor* c, std::vector<BcTaskView>& out, int* device);
void compressor_clear(bc_compressor* c);

}  // namespace bcn

using namespace bcn;

namespace {

struct Group {
    int kind;  // 0: BC1-BC5, 1: BC7 (shared settings), 2: one BC6H task
    uint32_t tile0, ntiles;
    BC7SettingsDev s7;
    BC6HSettingsDev s6;
    BcTaskView task;  // kind 2
};

int set_err(cudaError_t e) {
    record_cuda_error(e);
    return BC_ERR_CUDA;
}
#define BATCH_CUDA(call)                               \
    do {                                               \
        cudaError_t e_ = (call);                       \
        if (e_ != cudaSuccess) return set_err(e_);     \
    } while (0)

std::mutex g_tune_mu;
std::map<std::string, bc_tune> g_tune_cache;

}  // namespace

struct bc_batch {
    int device = 0;
    std::vector<Group> groups;
    uint32_t bc15_tiles = 0;
    TaskDesc* d_tasks = nullptr;
    uint32_t* d_tile_task = nullptr;
    uint32_t* d_counter = nullptr;
    void* d_scratch = nullptr;
    cudaGraphExec_t exec = nullptr;
    int sms = 148;
    bc_tune tune;
    std::string key;
};

namespace {

// Enqueues the whole batch (no graph) on `s` with launch shape `t`;
// `which` selects groups: -1 all, otherwise only groups of that kind.
int enqueue(bc_batch* b, const bc_tune& t, cudaStream_t s, int which) {
    for (const Group& g : b->groups) {
        if (which >= 0 && g.kind != which) continue;
        if (g.kind == 0) {
            BATCH_CUDA(cudaMemsetAsync(b->d_counter, 0, sizeof(uint32_t), s));
            int ctas = b->sms * (int)t.ctas_per_sm;
            BATCH_CUDA(launch_bc15_batch(b->d_tasks, b->d_tile_task + g.tile0, g.ntiles, b->d_counter,
                                         (int)t.threads_per_cta, ctas, (int)t.tiles_per_claim, s));
        } else if (g.kind == 1) {
            BATCH_CUDA(launch_bc7_batch(b->d_tasks, b->d_tile_task + g.tile0, g.ntiles, g.s7, b->d_scratch,
                                        (int)t.bc7_search_warps, s));
        } else {
            const BcTaskView& v = g.task;
            BATCH_CUDA(launch_bc6h_encode(v.src, v.pitch, BC6H_SRC_RGBA16F, (v.w + 3) / 4, (v.h + 3) / 4, v.dst,
                                          g.s6, b->d_scratch, s));
        }
    }
    return BC_OK;
}

int capture(bc_batch* b) {
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    // the BC7 pipeline's side streams must exist before capture begins
    BATCH_CUDA(bc7_side_streams_init());
    cudaStream_t cs;
    BATCH_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    int rc = BC_OK;
    if (e == cudaSuccess) {
        rc = enqueue(b, b->tune, cs, -1);
        cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
        if (rc == BC_OK && e2 != cudaSuccess) rc = set_err(e2);
    } else {
        rc = set_err(e);
    }
    if (rc == BC_OK) {
        e = cudaGraphInstantiate(&b->exec, graph, 0);
        if (e != cudaSuccess) rc = set_err(e);
    }
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cs);
    return rc;
}

// Times `which` groups of the batch under shape t: best of `reps` runs, ms.
int time_shape(bc_batch* b, const bc_tune& t, cudaStream_t s, int which, int reps, float* ms) {
    cudaEvent_t a, z;
    BATCH_CUDA(cudaEventCreate(&a));
    BATCH_CUDA(cudaEventCreate(&z));
    float best = 1e30f;
    int rc = enqueue(b, t, s, which);  // warm-up
    for (int r = 0; rc == BC_OK && r < reps; r++) {
        cudaEventRecord(a, s);
        rc = enqueue(b, t, s, which);
        cudaEventRecord(z, s);
        if (cudaEventSynchronize(z) != cudaSuccess) rc = BC_ERR_CUDA;
        float m = 0;
        cudaEventElapsedTime(&m, a, z);
        if (m < best) best = m;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(z);
    *ms = best;
    return rc;
}

int autotune(bc_batch* b, cudaStream_t s) {
    bc_tune best = b->tune;
    bool has15 = false, has7 = false;
    for (const Group& g : b->groups) {
        has15 |= g.kind == 0;
        has7 |= g.kind == 1;
    }
    if (has15) {
        float best_ms = 1e30f;
        const uint32_t threads[2] = {128, 256}, ctas[3] = {2, 4, 8}, claims[2] = {1, 4};
        for (uint32_t th : threads)
            for (uint32_t c : ctas)
                for (uint32_t cl : claims) {
                    bc_tune t = best;
                    t.threads_per_cta = th;
                    t.ctas_per_sm = c;
                    t.tiles_per_claim = cl;
                    float ms;
                    int rc = time_shape(b, t, s, 0, 2, &ms);
                    if (rc != BC_OK) return rc;
                    if (ms < best_ms) {
                        best_ms = ms;
                        best.threads_per_cta = th;
                        best.ctas_per_sm = c;
                        best.tiles_per_claim = cl;
                    }
                }
    }
    if (has7) {
        float best_ms = 1e30f;
        for (uint32_t sw : {4u, 8u}) {
            bc_tune t = best;
            t.bc7_search_warps = sw;
            float ms;
            int rc = time_shape(b, t, s, 1, 1, &ms);
            if (rc != BC_OK) return rc;
            if (ms < best_ms) {
                best_ms = ms;
                best.bc7_search_warps = sw;
            }
        }
    }
    b->tune = best;
    return BC_OK;
}

bool valid_tune(const bc_tune& t) {
    return (t.threads_per_cta == 128 || t.threads_per_cta == 256) && t.ctas_per_sm >= 1 && t.ctas_per_sm <= 16 &&
           t.tiles_per_claim >= 1 && t.tiles_per_claim <= 64 &&
           (t.bc7_search_warps == 4 || t.bc7_search_warps == 8);
}

}  // namespace

extern "C" int bc_batch_create(bc_compressor* c, const bc_tune* tune, int autotune_flag, void* stream,
                               bc_batch** out) {
    if (!c || !out) return BC_ERR_NULL;
    if (tune && !valid_tune(*tune)) return BC_ERR_SETTINGS;
    std::vector<BcTaskView> tasks;
    int device = 0;
    int rc = compressor_tasks(c, tasks, &device);
    if (rc != BC_OK) return rc;
    int prev = 0;
    BATCH_CUDA(cudaGetDevice(&prev));
    if (prev != device) BATCH_CUDA(cudaSetDevice(device));

    bc_batch* b = new bc_batch();
    b->device = device;
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device);
    std::vector<TaskDesc> descs;
    std::vector<uint32_t> tile_task;
    auto add_tiles = [&](const BcTaskView& v, int variant, uint32_t group_tile0) {
        TaskDesc d;
        memset(&d, 0, sizeof(d));
        d.src = v.src;
        d.dst = v.dst;
        d.stride = v.pitch;
        d.bw = (v.w + 3) / 4;
        d.bh = (v.h + 3) / 4;
        d.tile_base = (uint32_t)tile_task.size() - group_tile0;
        d.variant = (uint32_t)variant;
        d.aligned = ((uintptr_t)v.src % 16 == 0 && v.pitch % 16 == 0) ? 1u : 0u;
        uint32_t nt = (d.bw * d.bh + 31) / 32;
        uint32_t idx = (uint32_t)descs.size();
        descs.push_back(d);
        for (uint32_t i = 0; i < nt; i++) tile_task.push_back(idx);
    };
    // BC1-BC5: one group
    {
        Group g;
        memset(&g, 0, sizeof(g));
        g.kind = 0;
        g.tile0 = (uint32_t)tile_task.size();
        for (const BcTaskView& v : tasks)
            if (v.variant <= BC_BC5 && v.w > 0 && v.h > 0) add_tiles(v, v.variant, g.tile0);
        g.ntiles = (uint32_t)tile_task.size() - g.tile0;
        if (g.ntiles) b->groups.push_back(g);
        b->bc15_tiles = g.ntiles;
    }
    // BC7: one group per distinct settings value, in first-seen order
    std::vector<bool> used(tasks.size(), false);
    size_t max_scratch = 0;
    for (size_t i = 0; i < tasks.size(); i++) {
        if (tasks[i].variant != BC_BC7 || used[i] || tasks[i].w == 0 || tasks[i].h == 0) continue;
        Group g;
        memset(&g, 0, sizeof(g));
        g.kind = 1;
        g.s7 = *(const BC7SettingsDev*)tasks[i].settings;
        g.tile0 = (uint32_t)tile_task.size();
        for (size_t j = i; j < tasks.size(); j++) {
            if (tasks[j].variant != BC_BC7 || used[j] || tasks[j].w == 0 || tasks[j].h == 0) continue;
            if (memcmp(tasks[j].settings, &g.s7, sizeof(g.s7)) != 0) continue;
            used[j] = true;
            add_tiles(tasks[j], BC_BC7, g.tile0);
        }
        g.ntiles = (uint32_t)tile_task.size() - g.tile0;
        size_t need = bc7_scratch_bytes_tiles(g.ntiles, g.s7);
        if (need > max_scratch) max_scratch = need;
        b->groups.push_back(g);
    }
    // BC6H: one group per task
    for (const BcTaskView& v : tasks) {
        if (v.variant != BC_BC6H || v.w == 0 || v.h == 0) continue;
        Group g;
        memset(&g, 0, sizeof(g));
        g.kind = 2;
        g.s6 = *(const BC6HSettingsDev*)v.settings;
        g.task = v;
        size_t need = bc6h_scratch_bytes(((v.w + 3) / 4) * ((v.h + 3) / 4), g.s6);
        if (need > max_scratch) max_scratch = need;
        b->groups.push_back(g);
    }
    compressor_clear(c);

    auto fail = [&](int code) {
        bc_batch_destroy(b);
        if (prev != device) cudaSetDevice(prev);
        return code;
    };
    if (!descs.empty()) {
        if (cudaMalloc(&b->d_tasks, descs.size() * sizeof(TaskDesc)) != cudaSuccess ||
            cudaMalloc(&b->d_tile_task, tile_task.size() * sizeof(uint32_t)) != cudaSuccess)
            return fail(BC_ERR_CUDA);
        if (cudaMemcpy(b->d_tasks, descs.data(), descs.size() * sizeof(TaskDesc), cudaMemcpyHostToDevice) !=
                cudaSuccess ||
            cudaMemcpy(b->d_tile_task, tile_task.data(), tile_task.size() * sizeof(uint32_t),
                       cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(BC_ERR_CUDA);
    }
    if (cudaMalloc(&b->d_counter, sizeof(uint32_t)) != cudaSuccess) return fail(BC_ERR_CUDA);
    if (max_scratch && cudaMalloc(&b->d_scratch, max_scratch) != cudaSuccess) return fail(BC_ERR_CUDA);
    if (upload_bc6h_tables() != BC_OK) return fail(BC_ERR_CUDA);

    // launch shape: explicit > cached autotune result > autotune now > defaults
    b->tune = bc_tune{256, 4, 4, 8};
    char key[128];
    snprintf(key, sizeof(key), "dev%d:bc15=%u:bc7=%zu", device, b->bc15_tiles, tile_task.size() - b->bc15_tiles);
    b->key = key;
    if (tune) {
        b->tune = *tune;
    } else {
        bool cached = false;
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            auto it = g_tune_cache.find(b->key);
            if (it != g_tune_cache.end()) {
                b->tune = it->second;
                cached = true;
            }
        }
        if (!cached && autotune_flag) {
            int r = autotune(b, (cudaStream_t)stream);
            if (r != BC_OK) return fail(r);
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tune_cache[b->key] = b->tune;
        }
    }
    rc = capture(b);
    if (rc != BC_OK) return fail(rc);
    if (prev != device) cudaSetDevice(prev);
    *out = b;
    return BC_OK;
}

extern "C" int bc_batch_launch(bc_batch* b, void* stream) {
    if (!b || !b->exec) return BC_ERR_NULL;
    BATCH_CUDA(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
    return BC_OK;
}

extern "C" int bc_batch_get_tune(const bc_batch* b, bc_tune* out) {
    if (!b || !out) return BC_ERR_NULL;
    *out = b->tune;
    return BC_OK;
}

extern "C" int bc_batch_destroy(bc_batch* b) {
    if (!b) return BC_OK;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->d_tasks) cudaFree(b->d_tasks);
    if (b->d_tile_task) cudaFree(b->d_tile_task);
    if (b->d_counter) cudaFree(b->d_counter);
    if (b->d_scratch) cudaFree(b->d_scratch);
    delete b;
    return BC_OK;
}

extern "C" int bc_compressor_compress_batched(bc_compressor* c, void* stream, const bc_tune* tune) {
    bc_batch* b = nullptr;
    int rc = bc_batch_create(c, tune, tune ? 0 : 1, stream, &b);
    if (rc != BC_OK) return rc;
    rc = bc_batch_launch(b, stream);
    if (rc == BC_OK) {
        cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
        if (e != cudaSuccess) rc = set_err(e);
    }
    bc_batch_destroy(b);
    return rc;
}
