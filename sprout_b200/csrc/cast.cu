// GPU ray cast: closest hit and any hit over the 8-wide quantized BVH built in bvh8.cpp.
//
// Kernel design (sm_100a):
//  * Persistent warps with dynamic ray fetch: each warp keeps 32 rays in flight; whenever
//    at least Refill_threshold lanes have finished, the warp takes that many new ray indices
//    with one atomicAdd on the launch's work counter, so lanes stay busy although ray costs
//    differ by orders of magnitude (most rays of the benchmark leave the root box at once).
//  * Traversal follows the compressed-wide-BVH scheme of Ylitie, Karras and Laine (HPG 2017):
//    a node group (child base, hit bits) and a triangle group (triangle base, hit bits) per
//    lane, a per-lane stack of pending node groups, children visited in the ray-octant order
//    fixed at build time.  One step of the loop is one node (8 child boxes) or one triangle.
//  * Child boxes are 8-bit offsets from the node origin with a power-of-two scale, so a slab
//    distance is one FMA per bound: t = q * (scale / d) + (origin - o) / d.
//  * The triangle test is the reference's Möller-Trumbore (triangle_primitive_mt.inl:100-131)
//    with its operation order: cross products as in simd.inl:173-187 (AVX2 path: one product
//    rounded, one fused), dot products as in simd.inl:165-171 ((x + y) + z), and an IEEE
//    reciprocal of the determinant in place of the reference's rcpss + Newton step
//    (scalar.inl:67-71).  Every operation is an explicit _rn intrinsic so that nvcc does not
//    contract them; results are bit-identical to the CPU restatement in oracle/.
//  * A triangle is hit when the test passes with min_t <= t <= max_t and the hit point
//    o + t * d (one FMA per axis) lies within the triangle's bounds widened by the tree's hit
//    margin (2^-17 of the scene size).  The second condition never rejects a genuine hit; it
//    rejects the rounding noise the test returns for zero-area triangles, whose "hits" can lie
//    anywhere along the ray.  Closest hit returns, among all hit triangles, the one with the
//    smallest t, ties going to the smaller triangle index.  That choice is independent of
//    tree shape and traversal order, so any correct traversal returns the same triangle.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>

#include "bvh8.hpp"
#include "common.hpp"

namespace {

constexpr int      Block            = 128;
constexpr uint32_t Stack_size       = spb::Max_wide_depth;
constexpr uint32_t Refill_threshold = 8;
constexpr uint32_t Full_mask        = 0xFFFFFFFFu;

// Counter slots (2 words each: work counter, overflow count).  Slot 0 serves the device
// entry points, slots 1 and 2 the two streams of the host pipeline.
constexpr uint32_t Num_counter_slots = 3;

struct Ray_state {
    float    ox, oy, oz;
    float    dx, dy, dz;
    float    ix, iy, iz;
    float    tmin, tbest;
    float    u, v;
    uint32_t best_id;
    uint32_t oct_inv;
};

__device__ __forceinline__ float q_to_float(uint32_t word, uint32_t k) {
    // byte k of word as a float: (2^23 + b) - 2^23, exact.
    return __uint_as_float(__byte_perm(word, 0x4B000000u, 0x7650u | k)) - 8388608.f;
}

// Reciprocal of a direction component for the slab test; components below 2^-80 in
// magnitude are replaced by +-2^-80 so that every slab distance stays finite.
__device__ __forceinline__ float safe_rcp(float d) {
    float const tiny = 8.27180613e-25f;  // 2^-80
    float const m    = fabsf(d) < tiny ? copysignf(tiny, d) : d;
    return __frcp_rn(m);
}

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by,
                                      float bz) {
    return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

// cross(a, b) with the reference's AVX2 operation order (simd.inl:173-187).
__device__ __forceinline__ void cross3(float ax, float ay, float az, float bx, float by,
                                       float bz, float& rx, float& ry, float& rz) {
    rx = __fmaf_rn(bz, ay, -__fmul_rn(az, by));
    ry = __fmaf_rn(bx, az, -__fmul_rn(ax, bz));
    rz = __fmaf_rn(by, ax, -__fmul_rn(ay, bx));
}

// Möller-Trumbore with inclusive bounds (triangle_primitive_mt.inl:100-131).
__device__ __forceinline__ bool triangle_test(Ray_state const& r, float4 a, float4 e1, float4 e2,
                                              float tmax, float& t, float& u, float& v) {
    float const tx = __fsub_rn(r.ox, a.x);
    float const ty = __fsub_rn(r.oy, a.y);
    float const tz = __fsub_rn(r.oz, a.z);

    float px, py, pz;
    cross3(r.dx, r.dy, r.dz, e2.x, e2.y, e2.z, px, py, pz);
    float qx, qy, qz;
    cross3(tx, ty, tz, e1.x, e1.y, e1.z, qx, qy, qz);

    float const det = dot3(e1.x, e1.y, e1.z, px, py, pz);
    float const tvp = dot3(tx, ty, tz, px, py, pz);
    float const dqv = dot3(r.dx, r.dy, r.dz, qx, qy, qz);
    float const eqv = dot3(e2.x, e2.y, e2.z, qx, qy, qz);

    float const inv = __frcp_rn(det);

    u        = __fmul_rn(tvp, inv);
    v        = __fmul_rn(dqv, inv);
    t        = __fmul_rn(eqv, inv);
    float uv = __fadd_rn(u, v);

    return (u >= 0.f) & (u <= 1.f) & (v >= 0.f) & (uv <= 1.f) & (t >= r.tmin) & (t <= tmax);
}

// The hit point o + t * d lies within the triangle's bounds widened by margin.
__device__ __forceinline__ bool within_bounds(Ray_state const& r, float4 a, float4 e1, float4 e2,
                                              float t, float margin) {
    float const p[3]  = {__fmaf_rn(t, r.dx, r.ox), __fmaf_rn(t, r.dy, r.oy),
                         __fmaf_rn(t, r.dz, r.oz)};
    float const va[3] = {a.x, a.y, a.z};
    float const vb[3] = {__fadd_rn(a.x, e1.x), __fadd_rn(a.y, e1.y), __fadd_rn(a.z, e1.z)};
    float const vc[3] = {__fadd_rn(a.x, e2.x), __fadd_rn(a.y, e2.y), __fadd_rn(a.z, e2.z)};
    bool inside = true;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float const lo = __fsub_rn(fminf(va[k], fminf(vb[k], vc[k])), margin);
        float const hi = __fadd_rn(fmaxf(va[k], fmaxf(vb[k], vc[k])), margin);
        inside &= (p[k] >= lo) & (p[k] <= hi);
    }
    return inside;
}

// Intersects the ray with the 8 child boxes of a node; returns the hit bits (internal
// children in bits 24..31 permuted by the ray octant, leaf triangles in bits 0..23).
__device__ __forceinline__ uint32_t node_test(Ray_state const& r, uint4 const* __restrict__ node,
                                              uint32_t& child_base, uint32_t& tri_base,
                                              uint32_t& imask) {
    uint4 const w0 = __ldg(node + 0);
    uint4 const w1 = __ldg(node + 1);
    uint4 const w2 = __ldg(node + 2);
    uint4 const w3 = __ldg(node + 3);
    uint4 const w4 = __ldg(node + 4);

    float const sx = __uint_as_float((w0.w & 0xFFu) << 23);
    float const sy = __uint_as_float(((w0.w >> 8) & 0xFFu) << 23);
    float const sz = __uint_as_float(((w0.w >> 16) & 0xFFu) << 23);
    imask          = w0.w >> 24;
    child_base     = w1.x;
    tri_base       = w1.y;

    float const adjx = sx * r.ix;
    float const adjy = sy * r.iy;
    float const adjz = sz * r.iz;
    float const orgx = (__uint_as_float(w0.x) - r.ox) * r.ix;
    float const orgy = (__uint_as_float(w0.y) - r.oy) * r.iy;
    float const orgz = (__uint_as_float(w0.z) - r.oz) * r.iz;

    bool const negx = r.ix < 0.f;
    bool const negy = r.iy < 0.f;
    bool const negz = r.iz < 0.f;

    uint32_t const oct_inv4 = r.oct_inv * 0x01010101u;

    uint32_t hits = 0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        uint32_t const lox  = h ? w2.y : w2.x;
        uint32_t const loy  = h ? w2.w : w2.z;
        uint32_t const loz  = h ? w3.y : w3.x;
        uint32_t const hix  = h ? w3.w : w3.z;
        uint32_t const hiy  = h ? w4.y : w4.x;
        uint32_t const hiz  = h ? w4.w : w4.z;
        uint32_t const meta = h ? w1.w : w1.z;

        uint32_t const nx = negx ? hix : lox;
        uint32_t const fx = negx ? lox : hix;
        uint32_t const ny = negy ? hiy : loy;
        uint32_t const fy = negy ? loy : hiy;
        uint32_t const nz = negz ? hiz : loz;
        uint32_t const fz = negz ? loz : hiz;

        // Internal children have 24..31 in the low five meta bits (bits 3 and 4 set).
        uint32_t const is_inner   = (meta & (meta << 1)) & 0x10101010u;
        uint32_t const inner_mask = __vcmpne4(is_inner, 0u);
        uint32_t const bit_index4 = (meta ^ (oct_inv4 & inner_mask)) & 0x1F1F1F1Fu;
        uint32_t const child_bits = (meta >> 5) & 0x07070707u;

#pragma unroll
        for (uint32_t k = 0; k < 4; ++k) {
            float const tnx = fmaf(q_to_float(nx, k), adjx, orgx);
            float const tny = fmaf(q_to_float(ny, k), adjy, orgy);
            float const tnz = fmaf(q_to_float(nz, k), adjz, orgz);
            float const tfx = fmaf(q_to_float(fx, k), adjx, orgx);
            float const tfy = fmaf(q_to_float(fy, k), adjy, orgy);
            float const tfz = fmaf(q_to_float(fz, k), adjz, orgz);

            float const tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, r.tmin));
            float const tf = fminf(fminf(tfx, tfy), fminf(tfz, r.tbest));

            if (tn <= tf) {
                uint32_t const bits = (child_bits >> (8 * k)) & 0xFFu;
                uint32_t const idx  = (bit_index4 >> (8 * k)) & 0xFFu;
                hits |= bits << idx;
            }
        }
    }
    return hits;
}

template <bool Any_hit>
__global__ void __launch_bounds__(Block)
    cast_kernel(uint4 const* __restrict__ nodes, float4 const* __restrict__ triangles,
                float4 const* __restrict__ rays, uint32_t num_rays, uint32_t* __restrict__ ids,
                float* __restrict__ ts, float2* __restrict__ uvs, uint8_t* __restrict__ occluded,
                uint32_t* __restrict__ counters, float hit_margin) {
    uint32_t const lane = threadIdx.x & 31u;
    uint32_t const lt   = (1u << lane) - 1u;

    uint2 stack[Stack_size];
    uint32_t sp = 0;

    Ray_state r;
    uint2     group     = make_uint2(0, 0);
    uint2     tri_group = make_uint2(0, 0);
    uint32_t  ray       = 0;
    bool      active    = false;
    bool      exhausted = false;

    while (true) {
        uint32_t const idle = __ballot_sync(Full_mask, !active);
        if (exhausted && idle == Full_mask) {
            break;
        }
        if (!exhausted && __popc(idle) >= int(Refill_threshold)) {
            uint32_t const count  = __popc(idle);
            uint32_t const leader = __ffs(idle) - 1;
            uint32_t       base   = 0;
            if (lane == leader) {
                base = atomicAdd(counters, count);
            }
            base = __shfl_sync(Full_mask, base, leader);
            if (uint64_t(base) + count >= num_rays) {
                exhausted = true;
            }
            if (!active) {
                uint32_t const mine = base + __popc(idle & lt);
                if (mine < num_rays) {
                    ray              = mine;
                    float4 const ro  = __ldg(rays + 2 * size_t(mine));
                    float4 const rd  = __ldg(rays + 2 * size_t(mine) + 1);
                    r.ox             = ro.x;
                    r.oy             = ro.y;
                    r.oz             = ro.z;
                    r.tmin           = ro.w;
                    r.dx             = rd.x;
                    r.dy             = rd.y;
                    r.dz             = rd.z;
                    r.tbest          = rd.w;
                    r.ix             = safe_rcp(rd.x);
                    r.iy             = safe_rcp(rd.y);
                    r.iz             = safe_rcp(rd.z);
                    r.u              = 0.f;
                    r.v              = 0.f;
                    r.best_id        = SPB_MISS;
                    uint32_t const o = (r.ix < 0.f ? 1u : 0u) | (r.iy < 0.f ? 2u : 0u) |
                                       (r.iz < 0.f ? 4u : 0u);
                    r.oct_inv        = 7u - o;
                    group            = make_uint2(0, 0x80000000u);
                    tri_group        = make_uint2(0, 0);
                    sp               = 0;
                    active           = true;
                }
            }
        }

        if (!active) {
            continue;
        }

        bool done = false;
        if (tri_group.y != 0) {
            uint32_t const k = __ffs(tri_group.y) - 1;
            tri_group.y &= tri_group.y - 1;
            float4 const* tri = triangles + 3 * size_t(tri_group.x + k);
            float4 const  a   = __ldg(tri + 0);
            float4 const  e1  = __ldg(tri + 1);
            float4 const  e2  = __ldg(tri + 2);
            float         t, u, v;
            if (triangle_test(r, a, e1, e2, r.tbest, t, u, v) &&
                within_bounds(r, a, e1, e2, t, hit_margin)) {
                uint32_t const id = __float_as_uint(a.w);
                if (Any_hit) {
                    r.best_id = id;
                    done      = true;
                } else if (t < r.tbest || id < r.best_id) {
                    r.tbest   = t;
                    r.best_id = id;
                    r.u       = u;
                    r.v       = v;
                }
            }
        } else if (group.y & 0xFF000000u) {
            uint32_t const b = 31u - __clz(group.y & 0xFF000000u);
            group.y &= ~(1u << b);
            uint32_t const slot = (b - 24u) ^ r.oct_inv;
            uint32_t const rel  = __popc(group.y & 0xFFu & ((1u << slot) - 1u));
            uint32_t const node = group.x + rel;
            if (group.y & 0xFF000000u) {
                if (sp < Stack_size) {
                    stack[sp++] = group;
                } else {
                    atomicAdd(counters + 1, 1u);
                    r.best_id = SPB_MISS;
                    done      = true;
                }
            }
            if (!done) {
                uint32_t child_base, tri_base, imask;
                uint32_t const hits = node_test(r, nodes + 5 * size_t(node), child_base,
                                                tri_base, imask);
                group               = make_uint2(child_base, (hits & 0xFF000000u) | imask);
                tri_group           = make_uint2(tri_base, hits & 0x00FFFFFFu);
            }
        } else if (sp > 0) {
            group = stack[--sp];
        } else {
            done = true;
        }

        if (done) {
            if (Any_hit) {
                occluded[ray] = r.best_id != SPB_MISS ? 1 : 0;
            } else {
                ids[ray] = r.best_id;
                ts[ray]  = r.tbest;
                if (uvs) {
                    uvs[ray] = make_float2(r.u, r.v);
                }
            }
            active = false;
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
    bool          built      = false;
    float         hit_margin = 0.f;
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
            nullptr, nullptr, occ, counters, tree->hit_margin);
    } else {
        cast_kernel<false><<<grid, Block, 0, stream>>>(
            reinterpret_cast<uint4 const*>(tree->d_nodes), tree->d_tris, rays, n, ids, ts, uvs,
            nullptr, counters, tree->hit_margin);
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
    if (e != cudaSuccess) {
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
