// Device-side traversal of the 8-wide quantized BVH (bvh8.cpp), shared by the ray-cast
// entry points (cast.cu) and the path tracer's extend / shadow kernels (render.cu).
//
// Traversal follows the compressed-wide-BVH scheme of Ylitie, Karras and Laine (HPG 2017):
// a node group (child base, hit bits) and a triangle group (triangle base, hit bits) per
// lane, a per-lane stack of pending node groups, children visited in the ray-octant order
// fixed at build time.  One step is one node (8 child boxes) or one triangle.
//
// The triangle test is the reference's Möller-Trumbore (triangle_primitive_mt.inl:100-131)
// with its operation order: cross products as in simd.inl:173-187 (AVX2 path: one product
// rounded, one fused), dot products as in simd.inl:165-171 ((x + y) + z), and an IEEE
// reciprocal of the determinant in place of the reference's rcpss + Newton step
// (scalar.inl:67-71).  Every operation is an explicit _rn intrinsic so that nvcc does not
// contract them; results are bit-identical to the CPU restatement in oracle/.
//
// A triangle is hit when the test passes with min_t <= t <= max_t and the hit point
// o + t * d (one FMA per axis) lies within the triangle's bounds widened by the tree's hit
// margin (2^-17 of the scene size).  The second condition never rejects a genuine hit; it
// rejects the rounding noise the test returns for zero-area triangles, whose "hits" can lie
// anywhere along the ray.  Closest hit keeps, among all hit triangles, the one with the
// smallest t, ties going to the smaller triangle index: the answer does not depend on tree
// shape or traversal order.
#pragma once

#include <cstdint>

#include "bvh8.hpp"

namespace spb::gpu {

constexpr uint32_t Stack_size = Max_wide_depth;
constexpr uint32_t Miss       = 0xFFFFFFFFu;

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


// Whether the ray's [min_t, max_t] overlaps the box [lo, hi]: a slab test in double precision
// whose reciprocals are the ray's slab reciprocals (start_ray) refined by one Newton step, so
// that rounding cannot reject a ray that passes through the box by more than about 1e-14 of
// its distance to it.  A NaN anywhere makes the test pass (fmin and fmax ignore NaN), leaving
// such rays to the traversal.  Used with the tree's scene box (Wide_bvh::scene_lo/hi), which
// is padded by 128 hit margins: every ray it rejects ends as a miss of the full traversal too.
__device__ __forceinline__ bool enters_box(Ray_state const& r, float3 lo, float3 hi) {
    float const o[3]   = {r.ox, r.oy, r.oz};
    float const d[3]   = {r.dx, r.dy, r.dz};
    float const inv[3] = {r.ix, r.iy, r.iz};
    float const l[3]   = {lo.x, lo.y, lo.z};
    float const h[3]   = {hi.x, hi.y, hi.z};
    double      tn     = r.tmin;
    double      tf     = r.tbest;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float const  tiny = 8.27180613e-25f;  // 2^-80, as safe_rcp
        double const m    = fabsf(d[k]) < tiny ? copysignf(tiny, d[k]) : d[k];
        double       i    = inv[k];
        i                 = i * fma(-m, i, 2.0);
        double const a    = (double(l[k]) - double(o[k])) * i;
        double const b    = (double(h[k]) - double(o[k])) * i;
        tn                = fmax(tn, fmin(a, b));
        tf                = fmin(tf, fmax(a, b));
    }
    return tn <= tf;
}

// Per-lane traversal state kept in registers; the node-group stack itself is a separate
// array (local memory), so that dynamic indexing into it does not pull these scalars out of
// registers.
struct Traversal {
    uint2    group;      // node group: child base, internal-child hit bits << 24 | imask
    uint2    tri_group;  // triangle group: triangle base, triangle hit bits
    uint32_t sp;
};

// Loads one ray (math::ray order: origin, min_t / direction, max_t) and resets the state.
__device__ __forceinline__ void start_ray(Ray_state& r, Traversal& tv, float4 ro, float4 rd) {
    r.ox      = ro.x;
    r.oy      = ro.y;
    r.oz      = ro.z;
    r.tmin    = ro.w;
    r.dx      = rd.x;
    r.dy      = rd.y;
    r.dz      = rd.z;
    r.tbest   = rd.w;
    r.ix      = safe_rcp(rd.x);
    r.iy      = safe_rcp(rd.y);
    r.iz      = safe_rcp(rd.z);
    r.u       = 0.f;
    r.v       = 0.f;
    r.best_id = Miss;
    uint32_t const o = (r.ix < 0.f ? 1u : 0u) | (r.iy < 0.f ? 2u : 0u) | (r.iz < 0.f ? 4u : 0u);
    r.oct_inv        = 7u - o;
    tv.group         = make_uint2(0, 0x80000000u);  // the root, as the only child of a group
    tv.tri_group     = make_uint2(0, 0);
    tv.sp            = 0;
}

// ---- two-level traversal (instancing) ----
// The top-level tree's leaf records are instances (Wide_triangle::id = instance index).  A lane
// reaching one pushes what is left of its top-level traversal (pending node group, then pending
// leaves), transforms its ray into the instance's object space -- the direction by the linear
// part only, not renormalised, so that t is the same parameter in both spaces and min_t,
// the closest hit so far and every hit distance carry over -- and walks the instance's own tree
// from its root.  When that tree is spent (the stack back at the depth where it began), the
// world ray is restored and the top-level traversal resumes.  A stack entry whose top byte is
// zero is a group of pending top-level leaves (node groups are pushed only while they still
// have children to visit, in the top byte).

// What the traversal reads of an instance: its world-to-object map (rows: object_k =
// dot(row_k.xyz, world) + row_k.w), the root node of its tree and that tree's hit margin.
struct Instance_trace {
    float4   w2o[3];
    uint32_t root;
    float    hit_margin;
    uint32_t pad[2];
};
static_assert(sizeof(Instance_trace) == 64, "Instance_trace is 64 bytes");

// A lane's two-level state: the world-space ray, kept while the lane is inside an instance;
// the instance it is in (Miss at the top level); the stack depth at which that instance's tree
// began; the instance of the closest hit so far; the hit margin of the current tree.
struct Instance_state {
    float    wox, woy, woz;
    float    wdx, wdy, wdz;
    uint32_t inst;
    uint32_t base_sp;
    uint32_t best_inst;
    float    margin;
};

__device__ __forceinline__ void start_instances(Ray_state const& r, Instance_state& is) {
    is.wox       = r.ox;
    is.woy       = r.oy;
    is.woz       = r.oz;
    is.wdx       = r.dx;
    is.wdy       = r.dy;
    is.wdz       = r.dz;
    is.inst      = Miss;
    is.base_sp   = 0;
    is.best_inst = Miss;
    is.margin    = 0.f;
}

// The ray's origin and direction replaced (slab reciprocals and octant recomputed).
__device__ __forceinline__ void set_ray(Ray_state& r, float ox, float oy, float oz, float dx,
                                        float dy, float dz) {
    r.ox = ox;
    r.oy = oy;
    r.oz = oz;
    r.dx = dx;
    r.dy = dy;
    r.dz = dz;
    r.ix = safe_rcp(dx);
    r.iy = safe_rcp(dy);
    r.iz = safe_rcp(dz);
    uint32_t const o = (r.ix < 0.f ? 1u : 0u) | (r.iy < 0.f ? 2u : 0u) | (r.iz < 0.f ? 4u : 0u);
    r.oct_inv        = 7u - o;
}

__device__ __forceinline__ bool push_group(uint2* stack, Traversal& tv, uint2 group) {
    if (tv.sp < Stack_size) {
        stack[tv.sp++] = group;
        return true;
    }
    return false;
}

// One traversal step: a triangle if the current triangle group has one pending, else the
// next node (taking the next group from the stack when the current one is spent).
// Returns true when the ray is finished (any hit found, or nothing left to visit).
// overflow receives a count if the stack guard ever trips (it cannot for trees of depth
// <= Max_wide_depth, nor for two-level trees whose depths add up to at most that); the ray
// then ends as a miss instead of writing out of bounds.
// Filter: triangles whose class word (Wide_triangle::tri_class) shares a bit with skip_class
// are ignored (the path tracer skips medium boundaries for shadow rays, and surfaces when it
// walks the boundaries along a shadow ray).
// Instances: two-level traversal (is, instances); the top-level tree's leaves are instances.
template <bool Any_hit, bool Filter = false, bool Instances = false>
__device__ __forceinline__ bool traversal_step(Ray_state& r, Traversal& tv, uint2* stack,
                                               uint4 const* __restrict__ nodes,
                                               float4 const* __restrict__ triangles,
                                               float hit_margin, uint32_t* overflow,
                                               uint32_t skip_class = 0,
                                               Instance_state* is = nullptr,
                                               Instance_trace const* __restrict__ instances = nullptr) {
    // Single exit (no early return): the place where the two branches rejoin decides where a
    // diverged warp reconverges, and keeping it at the end measured fastest.
    bool done = false;
    if (tv.tri_group.y != 0) {
        uint32_t const k = __ffs(tv.tri_group.y) - 1;
        tv.tri_group.y &= tv.tri_group.y - 1;
        float4 const* tri = triangles + 3 * size_t(tv.tri_group.x + k);
        float4 const  a   = __ldg(tri + 0);
        bool          enter = false;
        if constexpr (Instances) {
            enter = is->inst == Miss;
        }
        if (enter) {
            if constexpr (Instances) {
                // A top-level leaf: keep the rest of the top-level traversal, enter the instance.
                uint32_t const inst = __float_as_uint(a.w);
                bool           ok   = true;
                if (tv.group.y & 0xFF000000u) {
                    ok = push_group(stack, tv, tv.group);
                }
                if (ok && tv.tri_group.y != 0) {
                    ok = push_group(stack, tv, tv.tri_group);
                }
                if (!ok) {
                    atomicAdd(overflow, 1u);
                    r.best_id = Miss;
                    done      = true;
                } else {
                    Instance_trace const& it = instances[inst];
                    float4 const          m0 = __ldg(&it.w2o[0]);
                    float4 const          m1 = __ldg(&it.w2o[1]);
                    float4 const          m2 = __ldg(&it.w2o[2]);
                    uint32_t const        root = __ldg(&it.root);
                    is->margin  = __ldg(&it.hit_margin);
                    is->inst    = inst;
                    is->base_sp = tv.sp;
                    set_ray(r, fmaf(m0.x, is->wox, fmaf(m0.y, is->woy, fmaf(m0.z, is->woz, m0.w))),
                            fmaf(m1.x, is->wox, fmaf(m1.y, is->woy, fmaf(m1.z, is->woz, m1.w))),
                            fmaf(m2.x, is->wox, fmaf(m2.y, is->woy, fmaf(m2.z, is->woz, m2.w))),
                            fmaf(m0.x, is->wdx, fmaf(m0.y, is->wdy, m0.z * is->wdz)),
                            fmaf(m1.x, is->wdx, fmaf(m1.y, is->wdy, m1.z * is->wdz)),
                            fmaf(m2.x, is->wdx, fmaf(m2.y, is->wdy, m2.z * is->wdz)));
                    tv.group     = make_uint2(root, 0x80000000u);
                    tv.tri_group = make_uint2(0, 0);
                }
            }
        } else {
            float4 const e1 = __ldg(tri + 1);
            float4 const e2 = __ldg(tri + 2);
            float        t, u, v;
            float        margin = hit_margin;
            if constexpr (Instances) {
                margin = is->margin;
            }
            bool const candidate = !Filter || !(__float_as_uint(e1.w) & skip_class);
            if (candidate && triangle_test(r, a, e1, e2, r.tbest, t, u, v) &&
                within_bounds(r, a, e1, e2, t, margin)) {
                uint32_t const id = __float_as_uint(a.w);
                if (Any_hit) {
                    r.best_id = id;
                    if constexpr (Instances) {
                        is->best_inst = is->inst;
                    }
                    done = true;
                } else {
                    // t <= the closest t so far; equal distances go to the smaller
                    // (instance, triangle) pair.
                    bool closer = t < r.tbest;
                    if constexpr (Instances) {
                        closer = closer || is->inst < is->best_inst ||
                                 (is->inst == is->best_inst && id < r.best_id);
                    } else {
                        closer = closer || id < r.best_id;
                    }
                    if (closer) {
                        r.tbest   = t;
                        r.best_id = id;
                        r.u       = u;
                        r.v       = v;
                        if constexpr (Instances) {
                            is->best_inst = is->inst;
                        }
                    }
                }
            }
        }
    } else {
        bool leaves = false;  // a group of pending top-level leaves came off the stack
        if (!(tv.group.y & 0xFF000000u)) {
            if constexpr (Instances) {
                if (is->inst != Miss && tv.sp == is->base_sp) {
                    // The instance's tree is spent: back to the world ray.
                    set_ray(r, is->wox, is->woy, is->woz, is->wdx, is->wdy, is->wdz);
                    is->inst = Miss;
                }
            }
            // A spent node group is replaced by the next one from the stack in the same step,
            // so no step is spent on the pop alone.
            if (tv.sp > 0) {
                uint2 const e = stack[--tv.sp];
                if (Instances && !(e.y & 0xFF000000u)) {
                    tv.tri_group = e;
                    leaves       = true;
                } else {
                    tv.group = e;
                }
            }
        }
        if (leaves) {
            // nothing more this step: the next one enters the first of those instances
        } else if (tv.group.y & 0xFF000000u) {
            uint32_t const b = 31u - __clz(tv.group.y & 0xFF000000u);
            tv.group.y &= ~(1u << b);
            uint32_t const slot = (b - 24u) ^ r.oct_inv;
            uint32_t const rel  = __popc(tv.group.y & 0xFFu & ((1u << slot) - 1u));
            uint32_t const node = tv.group.x + rel;
            if (tv.group.y & 0xFF000000u) {
                if (!push_group(stack, tv, tv.group)) {
                    atomicAdd(overflow, 1u);
                    r.best_id = Miss;
                    done      = true;
                }
            }
            if (!done) {
                uint32_t child_base, tri_base, imask;
                uint32_t const hits =
                    node_test(r, nodes + 5 * size_t(node), child_base, tri_base, imask);
                tv.group     = make_uint2(child_base, (hits & 0xFF000000u) | imask);
                tv.tri_group = make_uint2(tri_base, hits & 0x00FFFFFFu);
            }
        } else {
            done = true;
        }
    }
    return done;
}

}  // namespace spb::gpu
