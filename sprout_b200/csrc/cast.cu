// GPU ray cast: closest hit and any hit over the 8-wide quantized BVH built in bvh8.cpp.
//
// Kernel design (sm_100a):
//  * Persistent warps with dynamic ray fetch: each warp keeps 32 rays in flight; whenever
//    at least Refill_threshold lanes have finished, the warp takes that many new ray indices
//    with one atomicAdd on the launch's work counter, so lanes stay busy although ray costs
//    differ by orders of magnitude.
//  * A fetched ray is first tested against the tree's padded scene box (gpu::enters_box, in
//    double precision); one that misses it (72 % of the benchmark's rays) is answered as a
//    miss at once, without the 8-child test of the root node.
//  * Rays are loaded with evict-first hints and results stored with streaming stores, so the
//    512 MiB of benchmark rays do not push the tree (63 MiB) out of L2.
//  * Traversal, triangle test and hit definition: traverse.cuh.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>

#include "bvh8.hpp"
#include "common.hpp"
#include "traverse.cuh"

namespace {

using namespace spb;

// Launch shape: 128-thread blocks, registers bounded so that SPB_CAST_MIN_BLOCKS blocks fit on
// an SM (9: 56 registers, 36 warps; measured 3 % faster than the unbounded 64 registers and
// 6 % faster than 48 registers at 10 blocks); a warp refills once Refill_threshold of its lanes
// are idle (8 measured best against 4, 12 and 16).
#ifndef SPB_CAST_REFILL
#define SPB_CAST_REFILL 8
#endif
#ifndef SPB_CAST_MIN_BLOCKS
#define SPB_CAST_MIN_BLOCKS 9
#endif
constexpr int      Block            = 128;
constexpr uint32_t Refill_threshold = SPB_CAST_REFILL;
#if SPB_CAST_MIN_BLOCKS > 0
#define SPB_CAST_BOUNDS __launch_bounds__(Block, SPB_CAST_MIN_BLOCKS)
#else
#define SPB_CAST_BOUNDS __launch_bounds__(Block)
#endif
constexpr uint32_t Full_mask        = 0xFFFFFFFFu;

// Counter slots (2 words each: work counter, overflow count).  Slot 0 serves the device
// entry points, slots 1 and 2 the two streams of the host pipeline.
constexpr uint32_t Num_counter_slots = 3;

// Stats: also count, per ray, the node and triangle steps of its traversal (summed per warp
// into stats[0] and stats[1]); the counting variant is only launched by spb_cast_stats_device.
template <bool Any_hit, bool Stats = false>
__global__ void SPB_CAST_BOUNDS
    cast_kernel(uint4 const* __restrict__ nodes, float4 const* __restrict__ triangles,
                float4 const* __restrict__ rays, uint32_t num_rays, uint32_t* __restrict__ ids,
                float* __restrict__ ts, float2* __restrict__ uvs, uint8_t* __restrict__ occluded,
                uint32_t* __restrict__ work, uint32_t* __restrict__ overflow, float hit_margin,
                float3 scene_lo, float3 scene_hi, unsigned long long* __restrict__ stats) {
    uint32_t const lane = threadIdx.x & 31u;
    uint32_t const lt   = (1u << lane) - 1u;

    gpu::Ray_state r;
    gpu::Traversal tv;
    uint2          stack[gpu::Stack_size];
    uint32_t       ray       = 0;
    bool           active    = false;
    bool           exhausted = false;
    uint32_t       node_steps = 0;
    uint32_t       tri_steps  = 0;

    while (true) {
        uint32_t idle = __ballot_sync(Full_mask, !active);
        if (exhausted && idle == Full_mask) {
            break;
        }
        // Refill while enough lanes are idle.  A fetched ray that misses the scene box is
        // answered at once (a miss) and its lane stays idle for the next round of the loop.
        while (!exhausted && __popc(idle) >= int(Refill_threshold)) {
            uint32_t const count  = __popc(idle);
            uint32_t const leader = __ffs(idle) - 1;
            uint32_t       base   = 0;
            if (lane == leader) {
                base = atomicAdd(work, count);
            }
            base = __shfl_sync(Full_mask, base, leader);
            if (uint64_t(base) + count >= num_rays) {
                exhausted = true;
            }
            if (!active) {
                uint32_t const mine = base + __popc(idle & lt);
                if (mine < num_rays) {
                    // Rays are read once: evict-first loads keep them from displacing the
                    // tree's nodes and triangles in L2.
                    gpu::start_ray(r, tv, __ldcs(rays + 2 * size_t(mine)),
                                   __ldcs(rays + 2 * size_t(mine) + 1));
                    if (gpu::enters_box(r, scene_lo, scene_hi)) {
                        ray    = mine;
                        active = true;
                    } else if (Any_hit) {
                        __stcs(occluded + mine, uint8_t(0));
                    } else {
                        __stcs(ids + mine, gpu::Miss);
                        __stcs(ts + mine, r.tbest);
                        if (uvs) {
                            __stcs(uvs + mine, make_float2(0.f, 0.f));
                        }
                    }
                }
            }
            idle = __ballot_sync(Full_mask, !active);
        }

        if (!active) {
            continue;
        }

        if constexpr (Stats) {
            if (tv.tri_group.y != 0) {
                ++tri_steps;
            } else if ((tv.group.y & 0xFF000000u) || tv.sp > 0) {
                ++node_steps;
            }
        }
        if (gpu::traversal_step<Any_hit>(r, tv, stack, nodes, triangles, hit_margin, overflow)) {
            if (Any_hit) {
                __stcs(occluded + ray, uint8_t(r.best_id != gpu::Miss ? 1 : 0));
            } else {
                __stcs(ids + ray, r.best_id);
                __stcs(ts + ray, r.tbest);
                if (uvs) {
                    __stcs(uvs + ray, make_float2(r.u, r.v));
                }
            }
            active = false;
        }
    }
    if constexpr (Stats) {
        unsigned long long n = node_steps;
        unsigned long long t = tri_steps;
        for (int o = 16; o > 0; o >>= 1) {
            n += __shfl_down_sync(Full_mask, n, o);
            t += __shfl_down_sync(Full_mask, t, o);
        }
        if (lane == 0) {
            atomicAdd(stats + 0, n);
            atomicAdd(stats + 1, t);
        }
    }
}

struct Pipeline {
    static constexpr uint64_t Chunk = 1ull << 21;  // rays per chunk

    cudaStream_t streams[2] = {nullptr, nullptr};
    float4*      rays[2]    = {nullptr, nullptr};
    uint32_t*    ids[2]     = {nullptr, nullptr};
    float*       ts[2]      = {nullptr, nullptr};
    float2*      uvs[2]     = {nullptr, nullptr};
    uint8_t*     occ[2]     = {nullptr, nullptr};
    bool         ready      = false;
};

}  // namespace

struct spb_tree {
    int           device     = 0;
    int           num_sms    = 0;
    int           grid_hit   = 0;
    int           grid_any   = 0;
    uint4*        d_nodes    = nullptr;
    float4*       d_tris     = nullptr;
    uint32_t*     d_counters = nullptr;
    unsigned long long* d_stats = nullptr;  // node steps, triangle steps (spb_cast_stats_device)
    bool          built      = false;
    float         hit_margin = 0.f;
    float3        scene_lo   = {0.f, 0.f, 0.f};  // Wide_bvh::scene_lo / scene_hi
    float3        scene_hi   = {0.f, 0.f, 0.f};
    spb_tree_info info{};
    Pipeline      pipe;
    cudaStream_t  last_stream = nullptr;
};

namespace {

int32_t cuda_fail(cudaError_t e, char const* what) {
    return spb::fail(SPB_ERROR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define SPB_CUDA(call)                          \
    do {                                        \
        cudaError_t const e_ = (call);          \
        if (e_ != cudaSuccess) {                \
            return cuda_fail(e_, #call);        \
        }                                       \
    } while (0)

class Device_scope {
  public:
    explicit Device_scope(int device) {
        cudaGetDevice(&previous_);
        if (previous_ != device) {
            cudaSetDevice(device);
        }
        device_ = device;
    }
    ~Device_scope() {
        if (previous_ != device_) {
            cudaSetDevice(previous_);
        }
    }

  private:
    int previous_ = 0;
    int device_   = 0;
};

void free_pipeline(Pipeline& p) {
    for (int s = 0; s < 2; ++s) {
        cudaFree(p.rays[s]);
        cudaFree(p.ids[s]);
        cudaFree(p.ts[s]);
        cudaFree(p.uvs[s]);
        cudaFree(p.occ[s]);
        if (p.streams[s]) {
            cudaStreamDestroy(p.streams[s]);
        }
    }
    p = Pipeline();
}

int32_t ensure_pipeline(spb_tree* tree) {
    Pipeline& p = tree->pipe;
    if (p.ready) {
        return SPB_OK;
    }
    for (int s = 0; s < 2; ++s) {
        SPB_CUDA(cudaStreamCreateWithFlags(&p.streams[s], cudaStreamNonBlocking));
        SPB_CUDA(cudaMalloc(&p.rays[s], Pipeline::Chunk * 32));
        SPB_CUDA(cudaMalloc(&p.ids[s], Pipeline::Chunk * 4));
        SPB_CUDA(cudaMalloc(&p.ts[s], Pipeline::Chunk * 4));
        SPB_CUDA(cudaMalloc(&p.uvs[s], Pipeline::Chunk * 8));
        SPB_CUDA(cudaMalloc(&p.occ[s], Pipeline::Chunk));
    }
    p.ready = true;
    return SPB_OK;
}

int32_t launch(spb_tree* tree, bool any_hit, uint32_t slot, float4 const* rays, uint32_t n,
               uint32_t* ids, float* ts, float2* uvs, uint8_t* occ, cudaStream_t stream) {
    uint32_t* counters = tree->d_counters + 2 * slot;
    SPB_CUDA(cudaMemsetAsync(counters, 0, sizeof(uint32_t), stream));
    int const full = any_hit ? tree->grid_any : tree->grid_hit;
    int const need = int((uint64_t(n) + Block - 1) / Block);
    int const grid = std::max(1, std::min(full, need));
    if (any_hit) {
        cast_kernel<true><<<grid, Block, 0, stream>>>(
            reinterpret_cast<uint4 const*>(tree->d_nodes), tree->d_tris, rays, n, nullptr,
            nullptr, nullptr, occ, counters, counters + 1, tree->hit_margin, tree->scene_lo, tree->scene_hi, nullptr);
    } else {
        cast_kernel<false><<<grid, Block, 0, stream>>>(
            reinterpret_cast<uint4 const*>(tree->d_nodes), tree->d_tris, rays, n, ids, ts, uvs,
            nullptr, counters, counters + 1, tree->hit_margin, tree->scene_lo, tree->scene_hi, nullptr);
    }
    SPB_CUDA(cudaGetLastError());
    return SPB_OK;
}

void release_device(spb_tree* tree) {
    cudaFree(tree->d_nodes);
    cudaFree(tree->d_tris);
    tree->d_nodes = nullptr;
    tree->d_tris  = nullptr;
    tree->built   = false;
}

}  // namespace

extern "C" SPB_API int32_t spb_tree_create(spb_tree** out) {
    spb::clear_error();
    if (!out) {
        return spb::fail(SPB_ERROR_ARGUMENT, "spb_tree_create: out is null");
    }
    *out = nullptr;
    auto* tree = new spb_tree;
    cudaError_t e = cudaGetDevice(&tree->device);
    if (e == cudaSuccess) {
        e = cudaDeviceGetAttribute(&tree->num_sms, cudaDevAttrMultiProcessorCount, tree->device);
    }
    int per_sm_hit = 0;
    int per_sm_any = 0;
    if (e == cudaSuccess) {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_hit, cast_kernel<false>, Block,
                                                          0);
    }
    if (e == cudaSuccess) {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_any, cast_kernel<true>, Block,
                                                          0);
    }
    if (e == cudaSuccess) {
        e = cudaMalloc(&tree->d_counters, 2 * Num_counter_slots * sizeof(uint32_t));
    }
    if (e == cudaSuccess) {
        e = cudaMemset(tree->d_counters, 0, 2 * Num_counter_slots * sizeof(uint32_t));
    }
    if (e == cudaSuccess) {
        e = cudaMalloc(&tree->d_stats, 2 * sizeof(unsigned long long));
    }
    if (e != cudaSuccess) {
        cudaFree(tree->d_stats);
        cudaFree(tree->d_counters);
        delete tree;
        return cuda_fail(e, "spb_tree_create");
    }
    tree->grid_hit = std::max(1, per_sm_hit) * tree->num_sms;
    tree->grid_any = std::max(1, per_sm_any) * tree->num_sms;
    *out           = tree;
    return SPB_OK;
}

extern "C" SPB_API int32_t spb_tree_release(spb_tree* tree) {
    spb::clear_error();
    if (!tree) {
        return spb::fail(SPB_ERROR_ARGUMENT, "spb_tree_release: tree is null");
    }
    {
        Device_scope scope(tree->device);
        cudaDeviceSynchronize();
        release_device(tree);
        free_pipeline(tree->pipe);
        cudaFree(tree->d_counters);
        cudaFree(tree->d_stats);
    }
    delete tree;
    return SPB_OK;
}

extern "C" SPB_API int32_t spb_tree_build(spb_tree* tree, uint32_t num_vertices,
                                          uint32_t num_triangles, float const* positions,
                                          uint32_t const* indices, uint32_t num_threads) {
    spb::clear_error();
    if (!tree || !positions || !indices) {
        return spb::fail(SPB_ERROR_ARGUMENT, "spb_tree_build: null argument");
    }
    if (num_triangles == 0 || num_vertices == 0) {
        return spb::fail(SPB_ERROR_ARGUMENT, "spb_tree_build: empty mesh");
    }
    Device_scope scope(tree->device);

    auto const     t0 = std::chrono::steady_clock::now();
    spb::Wide_bvh  bvh;
    std::string    error;
    if (!spb::build_wide_bvh(num_vertices, num_triangles, positions, indices,
                             spb::resolve_threads(num_threads), bvh, error)) {
        return spb::fail(SPB_ERROR_ARGUMENT, "spb_tree_build: %s", error.c_str());
    }

    SPB_CUDA(cudaDeviceSynchronize());
    release_device(tree);
    size_t const node_bytes = bvh.nodes.size() * sizeof(spb::Wide_node);
    size_t const tri_bytes  = bvh.triangles.size() * sizeof(spb::Wide_triangle);
    SPB_CUDA(cudaMalloc(&tree->d_nodes, node_bytes));
    SPB_CUDA(cudaMalloc(&tree->d_tris, tri_bytes));
    SPB_CUDA(cudaMemcpy(tree->d_nodes, bvh.nodes.data(), node_bytes, cudaMemcpyHostToDevice));
    SPB_CUDA(cudaMemcpy(tree->d_tris, bvh.triangles.data(), tri_bytes, cudaMemcpyHostToDevice));

    auto const t1 = std::chrono::steady_clock::now();

    tree->info.num_triangles = num_triangles;
    tree->info.num_nodes     = uint32_t(bvh.nodes.size());
    tree->info.num_leaves    = bvh.num_leaves;
    tree->info.max_depth     = bvh.max_depth;
    tree->info.device_bytes  = node_bytes + tri_bytes;
    tree->info.build_seconds = std::chrono::duration<double>(t1 - t0).count();
    tree->info.sah_cost      = bvh.sah_cost;
    tree->hit_margin         = bvh.hit_margin;
    tree->scene_lo           = make_float3(bvh.scene_lo[0], bvh.scene_lo[1], bvh.scene_lo[2]);
    tree->scene_hi           = make_float3(bvh.scene_hi[0], bvh.scene_hi[1], bvh.scene_hi[2]);
    tree->built              = true;
    return SPB_OK;
}

extern "C" SPB_API int32_t spb_tree_info_get(spb_tree const* tree, spb_tree_info* info) {
    spb::clear_error();
    if (!tree || !info) {
        return spb::fail(SPB_ERROR_ARGUMENT, "spb_tree_info_get: null argument");
    }
    *info = tree->info;
    return SPB_OK;
}

namespace {

int32_t check_cast(spb_tree* tree, float const* rays, uint64_t n, bool outputs_ok,
                   char const* who) {
    if (!tree) {
        return spb::fail(SPB_ERROR_ARGUMENT, "%s: tree is null", who);
    }
    if (!tree->built) {
        return spb::fail(SPB_ERROR_STATE, "%s: tree has not been built", who);
    }
    if (n > SPB_MAX_RAYS_PER_CALL) {
        return spb::fail(SPB_ERROR_ARGUMENT, "%s: %llu rays exceed the per-call limit", who,
                         (unsigned long long)n);
    }
    if (n > 0 && (!rays || !outputs_ok)) {
        return spb::fail(SPB_ERROR_ARGUMENT, "%s: null buffer", who);
    }
    return SPB_OK;
}

}  // namespace

extern "C" SPB_API int32_t spb_intersect_device(spb_tree* tree, float const* rays,
                                                uint64_t num_rays, uint32_t* ids, float* ts,
                                                float* uvs, void* stream) {
    spb::clear_error();
    if (int32_t const s = check_cast(tree, rays, num_rays, ids && ts, "spb_intersect_device")) {
        return s;
    }
    if (num_rays == 0) {
        return SPB_OK;
    }
    Device_scope scope(tree->device);
    tree->last_stream = static_cast<cudaStream_t>(stream);
    return launch(tree, false, 0, reinterpret_cast<float4 const*>(rays), uint32_t(num_rays), ids,
                  ts, reinterpret_cast<float2*>(uvs), nullptr, tree->last_stream);
}

extern "C" SPB_API int32_t spb_intersect_p_device(spb_tree* tree, float const* rays,
                                                  uint64_t num_rays, uint8_t* occluded,
                                                  void* stream) {
    spb::clear_error();
    if (int32_t const s = check_cast(tree, rays, num_rays, occluded != nullptr,
                                     "spb_intersect_p_device")) {
        return s;
    }
    if (num_rays == 0) {
        return SPB_OK;
    }
    Device_scope scope(tree->device);
    tree->last_stream = static_cast<cudaStream_t>(stream);
    return launch(tree, true, 0, reinterpret_cast<float4 const*>(rays), uint32_t(num_rays),
                  nullptr, nullptr, nullptr, occluded, tree->last_stream);
}

extern "C" SPB_API int32_t spb_cast_stats_device(spb_tree* tree, float const* rays,
                                                 uint64_t num_rays, uint32_t* ids, float* ts,
                                                 void* stream, uint64_t* node_steps,
                                                 uint64_t* triangle_steps) {
    spb::clear_error();
    if (int32_t const s = check_cast(tree, rays, num_rays, ids && ts && node_steps && triangle_steps,
                                     "spb_cast_stats_device")) {
        return s;
    }
    if (!node_steps || !triangle_steps) {
        return spb::fail(SPB_ERROR_ARGUMENT, "spb_cast_stats_device: null counter");
    }
    *node_steps     = 0;
    *triangle_steps = 0;
    if (num_rays == 0) {
        return SPB_OK;
    }
    Device_scope       scope(tree->device);
    cudaStream_t const st = static_cast<cudaStream_t>(stream);
    tree->last_stream     = st;
    uint32_t* counters    = tree->d_counters;
    SPB_CUDA(cudaMemsetAsync(counters, 0, sizeof(uint32_t), st));
    SPB_CUDA(cudaMemsetAsync(tree->d_stats, 0, 2 * sizeof(unsigned long long), st));
    uint32_t const n    = uint32_t(num_rays);
    int const      grid = std::max(1, std::min(tree->grid_hit, int((uint64_t(n) + Block - 1) / Block)));
    cast_kernel<false, true><<<grid, Block, 0, st>>>(
        reinterpret_cast<uint4 const*>(tree->d_nodes), tree->d_tris,
        reinterpret_cast<float4 const*>(rays), n, ids, ts, nullptr, nullptr, counters,
        counters + 1, tree->hit_margin, tree->scene_lo, tree->scene_hi, tree->d_stats);
    SPB_CUDA(cudaGetLastError());
    unsigned long long host[2] = {0, 0};
    SPB_CUDA(cudaMemcpyAsync(host, tree->d_stats, sizeof(host), cudaMemcpyDeviceToHost, st));
    SPB_CUDA(cudaStreamSynchronize(st));
    *node_steps     = host[0];
    *triangle_steps = host[1];
    return SPB_OK;
}

namespace {

int32_t cast_host(spb_tree* tree, bool any_hit, float const* rays, uint64_t n, uint32_t* ids,
                  float* ts, float* uvs, uint8_t* occ) {
    Device_scope scope(tree->device);
    if (int32_t const s = ensure_pipeline(tree)) {
        return s;
    }
    Pipeline& p = tree->pipe;
    uint64_t const chunks = (n + Pipeline::Chunk - 1) / Pipeline::Chunk;
    for (uint64_t c = 0; c < chunks; ++c) {
        int const          s     = int(c & 1);
        uint64_t const     first = c * Pipeline::Chunk;
        uint64_t const     count = std::min<uint64_t>(Pipeline::Chunk, n - first);
        cudaStream_t const st    = p.streams[s];
        SPB_CUDA(cudaMemcpyAsync(p.rays[s], rays + 8 * first, count * 32, cudaMemcpyHostToDevice,
                                 st));
        if (int32_t const r = launch(tree, any_hit, 1 + uint32_t(s), p.rays[s], uint32_t(count),
                                     p.ids[s], p.ts[s], uvs ? p.uvs[s] : nullptr, p.occ[s], st)) {
            return r;
        }
        if (any_hit) {
            SPB_CUDA(cudaMemcpyAsync(occ + first, p.occ[s], count, cudaMemcpyDeviceToHost, st));
        } else {
            SPB_CUDA(cudaMemcpyAsync(ids + first, p.ids[s], count * 4, cudaMemcpyDeviceToHost,
                                     st));
            SPB_CUDA(cudaMemcpyAsync(ts + first, p.ts[s], count * 4, cudaMemcpyDeviceToHost, st));
            if (uvs) {
                SPB_CUDA(cudaMemcpyAsync(uvs + 2 * first, p.uvs[s], count * 8,
                                         cudaMemcpyDeviceToHost, st));
            }
        }
    }
    SPB_CUDA(cudaStreamSynchronize(p.streams[0]));
    SPB_CUDA(cudaStreamSynchronize(p.streams[1]));
    tree->last_stream = p.streams[1];
    return SPB_OK;
}

}  // namespace

extern "C" SPB_API int32_t spb_intersect_host(spb_tree* tree, float const* rays,
                                              uint64_t num_rays, uint32_t* ids, float* ts,
                                              float* uvs) {
    spb::clear_error();
    if (int32_t const s = check_cast(tree, rays, num_rays, ids && ts, "spb_intersect_host")) {
        return s;
    }
    if (num_rays == 0) {
        return SPB_OK;
    }
    return cast_host(tree, false, rays, num_rays, ids, ts, uvs, nullptr);
}

extern "C" SPB_API int32_t spb_intersect_p_host(spb_tree* tree, float const* rays,
                                                uint64_t num_rays, uint8_t* occluded) {
    spb::clear_error();
    if (int32_t const s = check_cast(tree, rays, num_rays, occluded != nullptr,
                                     "spb_intersect_p_host")) {
        return s;
    }
    if (num_rays == 0) {
        return SPB_OK;
    }
    return cast_host(tree, true, rays, num_rays, nullptr, nullptr, nullptr, occluded);
}

extern "C" SPB_API int32_t spb_tree_status(spb_tree* tree, uint32_t* overflowed_rays) {
    spb::clear_error();
    if (!tree || !overflowed_rays) {
        return spb::fail(SPB_ERROR_ARGUMENT, "spb_tree_status: null argument");
    }
    Device_scope scope(tree->device);
    SPB_CUDA(cudaDeviceSynchronize());
    uint32_t host[2 * Num_counter_slots];
    SPB_CUDA(cudaMemcpy(host, tree->d_counters, sizeof(host), cudaMemcpyDeviceToHost));
    *overflowed_rays = host[1] + host[3] + host[5];
    return SPB_OK;
}

// ---- Closest hit without any device allocation ------------------------------------------
//
// Some callers cannot call cudaMalloc: a cudaMalloc may synchronize the whole device and may
// fail once device memory is exhausted, so a frame loop with a fixed time budget, or a host
// application whose own allocator owns all device memory, must not allocate on the way to a
// cast.  spb_intersect_host allocates device staging buffers on its first call;
// spb_intersect_host_static instead stages rays and results in the file-scope array below,
// which every GPU that loads this library holds until the process exits.

namespace {

constexpr uint64_t Static_max_rays      = SPB_STATIC_MAX_RAYS;
constexpr size_t   Static_counter_bytes = 256;  // work counter, padded
constexpr size_t   Static_scratch_bytes = Static_counter_bytes + Static_max_rays * (32 + 4 + 4);
constexpr int      Static_max_devices   = 64;

__device__ __align__(256) unsigned char g_static_scratch[Static_scratch_bytes];

// The array's device address per device, with the id of the CUDA context it was looked up in:
// a context created after a cudaDeviceReset may place the array elsewhere, so the address is
// looked up again whenever the current context's id differs from the cached one.
struct Static_address {
    unsigned char*     address    = nullptr;
    unsigned long long context_id = 0;
};

std::mutex     g_static_mutex;
Static_address g_static_address[Static_max_devices];

using Ctx_get_current = CUresult(CUDAAPI*)(CUcontext*);
using Ctx_get_id      = CUresult(CUDAAPI*)(CUcontext, unsigned long long*);

// Id of the calling thread's current context (0 if the driver cannot tell, in which case the
// address is looked up on every call).
unsigned long long current_context_id() {
    static Ctx_get_current get_current = nullptr;
    static Ctx_get_id      get_id      = nullptr;
    static bool const      resolved    = [] {
        void* a = nullptr;
        void* b = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault) == cudaSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault) == cudaSuccess) {
            get_current = reinterpret_cast<Ctx_get_current>(a);
            get_id      = reinterpret_cast<Ctx_get_id>(b);
        }
        return true;
    }();
    (void)resolved;
    CUcontext          ctx = nullptr;
    unsigned long long id  = 0;
    if (get_current && get_id && get_current(&ctx) == CUDA_SUCCESS && ctx &&
        get_id(ctx, &id) == CUDA_SUCCESS) {
        return id;
    }
    return 0;
}

// Device address of g_static_scratch on the current device, looked up once per device and
// context (the host-side symbol g_static_scratch itself is not a device address).
int32_t static_scratch(int device, unsigned char** out) {
    if (device < 0 || device >= Static_max_devices) {
        return spb::fail(SPB_ERROR_STATE, "spb_intersect_host_static: device %d not supported",
                         device);
    }
    unsigned long long const    context = current_context_id();
    std::lock_guard<std::mutex> lock(g_static_mutex);
    Static_address&             cached = g_static_address[device];
    if (!cached.address || context == 0 || cached.context_id != context) {
        void*             ptr = nullptr;
        cudaError_t const e   = cudaGetSymbolAddress(&ptr, g_static_scratch);
        if (e != cudaSuccess) {
            return cuda_fail(e, "cudaGetSymbolAddress(g_static_scratch)");
        }
        cached.address    = static_cast<unsigned char*>(ptr);
        cached.context_id = context;
    }
    *out = cached.address;
    return SPB_OK;
}

}  // namespace

extern "C" SPB_API int32_t spb_intersect_host_static(spb_tree* tree, float const* rays,
                                                     uint64_t num_rays, uint32_t* ids,
                                                     float* ts) {
    spb::clear_error();
    if (int32_t const s = check_cast(tree, rays, num_rays, ids && ts,
                                     "spb_intersect_host_static")) {
        return s;
    }
    if (num_rays > Static_max_rays) {
        return spb::fail(SPB_ERROR_ARGUMENT,
                         "spb_intersect_host_static: %llu rays exceed the static scratch limit "
                         "of %llu rays per call",
                         (unsigned long long)num_rays, (unsigned long long)Static_max_rays);
    }
    if (num_rays == 0) {
        return SPB_OK;
    }
    Device_scope scope(tree->device);
    unsigned char* base = nullptr;
    if (int32_t const s = static_scratch(tree->device, &base)) {
        return s;
    }
    auto* work   = reinterpret_cast<uint32_t*>(base);
    auto* d_rays = reinterpret_cast<float4*>(base + Static_counter_bytes);
    auto* d_ids  = reinterpret_cast<uint32_t*>(base + Static_counter_bytes + Static_max_rays * 32);
    auto* d_ts   = reinterpret_cast<float*>(base + Static_counter_bytes + Static_max_rays * 36);
    uint32_t const n = uint32_t(num_rays);

    // The array keeps the previous call's contents: the work counter must start at zero.
    // Stack overflows (none for trees this library builds) are counted in the tree's own
    // counter, as spb_intersect_host counts them, and reported by spb_tree_status.
    SPB_CUDA(cudaMemsetAsync(work, 0, sizeof(uint32_t), nullptr));
    SPB_CUDA(cudaMemcpyAsync(d_rays, rays, size_t(n) * 32, cudaMemcpyHostToDevice, nullptr));
    int const grid = std::max(1, std::min(tree->grid_hit, int((n + Block - 1) / Block)));
    cast_kernel<false><<<grid, Block, 0, nullptr>>>(reinterpret_cast<uint4 const*>(tree->d_nodes),
                                                    tree->d_tris, d_rays, n, d_ids, d_ts, nullptr,
                                                    nullptr, work, tree->d_counters + 1,
                                                    tree->hit_margin, tree->scene_lo, tree->scene_hi, nullptr);
    SPB_CUDA(cudaGetLastError());
    SPB_CUDA(cudaMemcpyAsync(ids, d_ids, size_t(n) * 4, cudaMemcpyDeviceToHost, nullptr));
    SPB_CUDA(cudaMemcpyAsync(ts, d_ts, size_t(n) * 4, cudaMemcpyDeviceToHost, nullptr));
    SPB_CUDA(cudaStreamSynchronize(nullptr));
    return SPB_OK;
}
