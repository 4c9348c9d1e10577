/*
 * CPU restatement of the reference's triangle-mesh ray cast.
 * TEST INFRASTRUCTURE ONLY: the parity tests, smoke check and the bench's CPU-baseline leg
 * use it as the checker; the product never links or calls it.
 *
 * What it restates (paths relative to the reference project, Opioid/sprout):
 *   - Möller-Trumbore with inclusive bounds, as the SSE path
 *     source/core/scene/shape/triangle/triangle_primitive_mt.inl:100-131
 *     (u >= 0, u <= 1, v >= 0, u + v <= 1, t >= min_t, t <= max_t; NaN fails every test);
 *   - its cross product in the operation order of source/base/math/simd.inl:173-187 on an
 *     AVX2 build (one product rounded, the other fused: fmaf), and its dot product
 *     ((x + y) + z) from simd.inl:165-171;
 *   - the closest-hit loop of Tree::intersect
 *     (source/core/scene/shape/triangle/bvh/triangle_bvh_tree.cpp:41-90): a triangle replaces
 *     the current hit when its t is <= the current max_t, and max_t shrinks to that t;
 *   - the any-hit loop of Tree::intersect_p (triangle_bvh_tree.cpp:145-185).
 *
 * A triangle counts as hit only when, in addition, the hit point o + t * d (fmaf per axis)
 * lies within the triangle's bounds (a, a + (b - a), a + (c - a)) widened by the hit margin
 * 2^-17 * max(scene extent, largest |coordinate|).  This never rejects a genuine hit; it
 * removes the rounding noise the test returns for zero-area triangles, whose "hits" can lie
 * anywhere along the ray (the reference's answer for those depends on its tree).
 *
 * Two deliberate, documented differences from the compiled reference:
 *   1. 1/det is the IEEE quotient 1.0f/det.  The reference uses rcpss plus one Newton step
 *      (source/base/math/scalar.inl:67-71), whose result depends on the CPU vendor's rcp
 *      table; u, v, t can differ in the last bit, which changes the outcome only for rays
 *      passing within rounding distance of a triangle edge.
 *   2. Ties: among triangles with the same t the smaller caller index wins (the reference
 *      keeps the last one tested in its tree order).  With this rule the answer does not
 *      depend on the tree at all: it is the minimum of (t, index) over every triangle that
 *      passes the test, which this oracle computes with a conservative BVH (padded boxes,
 *      double-precision slabs) or by brute force.
 *
 * Build: gcc -O2 -ffp-contract=off -fPIC -shared -pthread cast_oracle.c -o libcast_oracle.so -lm
 */
#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MISS 0xFFFFFFFFu

typedef struct {
    double lo[3];
    double hi[3];
    uint32_t left;  /* left child, or first primitive of a leaf */
    uint32_t right; /* right child */
    uint32_t count; /* primitives in a leaf, 0 for an inner node */
} Node;

typedef struct {
    uint32_t num_tris;
    float const* pos;
    uint32_t const* idx;
    Node* nodes;
    uint32_t* prims;
    double* cent;
    double* blo;
    double* bhi;
    uint32_t num_nodes;
    double pad;
    float margin;
} Tree;

typedef struct {
    double key;
    uint32_t prim;
} Sort_item;

static float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    float const x = ax * bx;
    float const y = ay * by;
    float const z = az * bz;
    float const s = x + y;
    return s + z;
}

static void cross3(float ax, float ay, float az, float bx, float by, float bz, float* r) {
    r[0] = fmaf(bz, ay, -(az * by));
    r[1] = fmaf(bx, az, -(ax * bz));
    r[2] = fmaf(by, ax, -(ay * bx));
}

/* Returns 1 if the triangle passes; t, u, v receive the computed values either way. */
static int mt_test(float const* ray, float const* a, float const* b, float const* c, float tmax,
                   float* t, float* u, float* v) {
    float e1[3], e2[3], tv[3], p[3], q[3];
    for (int k = 0; k < 3; ++k) {
        e1[k] = b[k] - a[k];
        e2[k] = c[k] - a[k];
        tv[k] = ray[k] - a[k];
    }
    cross3(ray[4], ray[5], ray[6], e2[0], e2[1], e2[2], p);
    cross3(tv[0], tv[1], tv[2], e1[0], e1[1], e1[2], q);

    float const det = dot3(e1[0], e1[1], e1[2], p[0], p[1], p[2]);
    float const tvp = dot3(tv[0], tv[1], tv[2], p[0], p[1], p[2]);
    float const dqv = dot3(ray[4], ray[5], ray[6], q[0], q[1], q[2]);
    float const eqv = dot3(e2[0], e2[1], e2[2], q[0], q[1], q[2]);

    float const inv = 1.0f / det;

    *u = tvp * inv;
    *v = dqv * inv;
    *t = eqv * inv;
    float const uv = *u + *v;

    return (*u >= 0.f) & (*u <= 1.f) & (*v >= 0.f) & (uv <= 1.f) & (*t >= ray[3]) &
           (*t <= tmax);
}

static int within_bounds(float const* ray, float const* a, float const* b, float const* c,
                         float t, float margin) {
    int inside = 1;
    for (int k = 0; k < 3; ++k) {
        float const e1 = b[k] - a[k];
        float const e2 = c[k] - a[k];
        float const vb = a[k] + e1;
        float const vc = a[k] + e2;
        float const p = fmaf(t, ray[4 + k], ray[k]);
        float lo = a[k] < vb ? a[k] : vb;
        float hi = a[k] > vb ? a[k] : vb;
        lo = vc < lo ? vc : lo;
        hi = vc > hi ? vc : hi;
        inside &= (p >= lo - margin) & (p <= hi + margin);
    }
    return inside;
}

/* The mesh's hit margin: 2^-17 * max(extent, magnitude) of the float vertex bounds. */
static float hit_margin_of(uint32_t num_triangles, float const* pos, uint32_t const* idx) {
    float lo[3] = {INFINITY, INFINITY, INFINITY};
    float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint64_t i = 0; i < 3 * (uint64_t)num_triangles; ++i) {
        float const* p = pos + 3 * (size_t)idx[i];
        for (int k = 0; k < 3; ++k) {
            if (p[k] < lo[k]) lo[k] = p[k];
            if (p[k] > hi[k]) hi[k] = p[k];
        }
    }
    double extent = 0.0, magnitude = 0.0;
    for (int k = 0; k < 3; ++k) {
        double const e = (double)hi[k] - (double)lo[k];
        if (e > extent) extent = e;
        if (fabs((double)lo[k]) > magnitude) magnitude = fabs((double)lo[k]);
        if (fabs((double)hi[k]) > magnitude) magnitude = fabs((double)hi[k]);
    }
    float const m = (float)ldexp(extent > magnitude ? extent : magnitude, -17);
    return m > FLT_MIN ? m : FLT_MIN;
}

static void tri_verts(Tree const* tr, uint32_t i, float const** a, float const** b,
                      float const** c) {
    *a = tr->pos + 3 * (size_t)tr->idx[3 * (size_t)i + 0];
    *b = tr->pos + 3 * (size_t)tr->idx[3 * (size_t)i + 1];
    *c = tr->pos + 3 * (size_t)tr->idx[3 * (size_t)i + 2];
}

/* ---- conservative BVH: median split on the longest centroid axis, <= 4 per leaf ---- */

static int cmp_item(void const* x, void const* y) {
    Sort_item const* a = (Sort_item const*)x;
    Sort_item const* b = (Sort_item const*)y;
    if (a->key < b->key) return -1;
    if (a->key > b->key) return 1;
    return (a->prim < b->prim) ? -1 : (a->prim > b->prim);
}

static uint32_t build_node(Tree* tr, Sort_item* scratch, uint32_t begin, uint32_t end) {
    uint32_t const id = tr->num_nodes++;
    Node* n = &tr->nodes[id];
    double clo[3] = {INFINITY, INFINITY, INFINITY};
    double chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int k = 0; k < 3; ++k) {
        n->lo[k] = INFINITY;
        n->hi[k] = -INFINITY;
    }
    for (uint32_t i = begin; i < end; ++i) {
        uint32_t const p = tr->prims[i];
        for (int k = 0; k < 3; ++k) {
            if (tr->blo[3 * (size_t)p + k] < n->lo[k]) n->lo[k] = tr->blo[3 * (size_t)p + k];
            if (tr->bhi[3 * (size_t)p + k] > n->hi[k]) n->hi[k] = tr->bhi[3 * (size_t)p + k];
            double const c = tr->cent[3 * (size_t)p + k];
            if (c < clo[k]) clo[k] = c;
            if (c > chi[k]) chi[k] = c;
        }
    }
    for (int k = 0; k < 3; ++k) {
        n->lo[k] -= tr->pad;
        n->hi[k] += tr->pad;
    }
    n->count = 0;
    if (end - begin <= 4) {
        n->left = begin;
        n->right = 0;
        n->count = end - begin;
        return id;
    }
    int axis = 0;
    for (int k = 1; k < 3; ++k) {
        if (chi[k] - clo[k] > chi[axis] - clo[axis]) axis = k;
    }
    for (uint32_t i = begin; i < end; ++i) {
        scratch[i].prim = tr->prims[i];
        scratch[i].key = tr->cent[3 * (size_t)tr->prims[i] + axis];
    }
    qsort(scratch + begin, end - begin, sizeof(Sort_item), cmp_item);
    for (uint32_t i = begin; i < end; ++i) {
        tr->prims[i] = scratch[i].prim;
    }
    uint32_t const mid = begin + (end - begin) / 2;
    uint32_t const l = build_node(tr, scratch, begin, mid);
    uint32_t const r = build_node(tr, scratch, mid, end);
    tr->nodes[id].left = l;
    tr->nodes[id].right = r;
    return id;
}

static int box_hit(Node const* n, double const* o, double const* inv, double tmin, double tmax) {
    double t0 = tmin;
    double t1 = tmax;
    for (int k = 0; k < 3; ++k) {
        double a = (n->lo[k] - o[k]) * inv[k];
        double b = (n->hi[k] - o[k]) * inv[k];
        if (isnan(a) || isnan(b)) {
            /* direction component 0 and origin on the slab plane: inside the slab */
            if (o[k] < n->lo[k] || o[k] > n->hi[k]) return 0;
            continue;
        }
        if (a > b) {
            double const s = a;
            a = b;
            b = s;
        }
        if (a > t0) t0 = a;
        if (b < t1) t1 = b;
    }
    return t0 <= t1;
}

typedef struct {
    Tree const* tr;
    float const* rays;
    uint64_t begin;
    uint64_t end;
    uint32_t* ids;
    float* ts;
    float* uvs;
    uint8_t* occ;
    int mode;
} Job;

static void cast_one(Tree const* tr, float const* ray, int any, int brute, uint32_t* id_out,
                     float* t_out, float* u_out, float* v_out) {
    float tbest = ray[7];
    uint32_t best = MISS;
    float bu = 0.f, bv = 0.f;

    if (brute) {
        for (uint32_t i = 0; i < tr->num_tris; ++i) {
            float const *a, *b, *c;
            float t, u, v;
            tri_verts(tr, i, &a, &b, &c);
            if (mt_test(ray, a, b, c, tbest, &t, &u, &v) &&
                within_bounds(ray, a, b, c, t, tr->margin)) {
                if (any) {
                    best = i;
                    break;
                }
                if (t < tbest || i < best) {
                    tbest = t;
                    best = i;
                    bu = u;
                    bv = v;
                }
            }
        }
    } else {
        double o[3], inv[3];
        for (int k = 0; k < 3; ++k) {
            o[k] = ray[k];
            inv[k] = 1.0 / (double)ray[4 + k];
        }
        uint32_t stack[256];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            uint32_t const ni = stack[--sp];
            Node const* n = &tr->nodes[ni];
            /* tmax of the box test: the current best, widened slightly for equal-t ties */
            if (!box_hit(n, o, inv, (double)ray[3], (double)tbest * (1.0 + 1e-6) + 1e-30)) {
                continue;
            }
            if (n->count > 0) {
                for (uint32_t k = 0; k < n->count; ++k) {
                    uint32_t const i = tr->prims[n->left + k];
                    float const *a, *b, *c;
                    float t, u, v;
                    tri_verts(tr, i, &a, &b, &c);
                    if (mt_test(ray, a, b, c, tbest, &t, &u, &v) &&
                within_bounds(ray, a, b, c, t, tr->margin)) {
                        if (any) {
                            best = i;
                            sp = 0;
                            break;
                        }
                        if (t < tbest || i < best) {
                            tbest = t;
                            best = i;
                            bu = u;
                            bv = v;
                        }
                    }
                }
            } else {
                if (sp + 2 > 256) {
                    abort();
                }
                stack[sp++] = n->right;
                stack[sp++] = n->left;
            }
        }
    }
    *id_out = best;
    *t_out = tbest;
    *u_out = bu;
    *v_out = bv;
}

static void* run_job(void* arg) {
    Job const* j = (Job const*)arg;
    int const brute = (j->mode & 4) != 0;
    for (uint64_t r = j->begin; r < j->end; ++r) {
        float const* ray = j->rays + 8 * r;
        uint32_t id;
        float t, u, v;
        if (j->mode & 1) {
            cast_one(j->tr, ray, 0, brute, &id, &t, &u, &v);
            j->ids[r] = id;
            j->ts[r] = t;
            if (j->uvs) {
                j->uvs[2 * r] = u;
                j->uvs[2 * r + 1] = v;
            }
        }
        if (j->mode & 2) {
            cast_one(j->tr, ray, 1, brute, &id, &t, &u, &v);
            j->occ[r] = id != MISS ? 1 : 0;
        }
    }
    return 0;
}

/*
 * mode: bit 0 closest hit (ids, ts, optional uvs), bit 1 any hit (occ),
 *       bit 2 brute force over all triangles instead of the BVH.
 * Returns 0, or -1 on bad arguments.
 */
int32_t oracle_cast(uint32_t num_vertices, uint32_t num_triangles, float const* positions,
                    uint32_t const* indices, uint64_t num_rays, float const* rays, uint32_t* ids,
                    float* ts, float* uvs, uint8_t* occ, uint32_t num_threads, int32_t mode) {
    if (!positions || !indices || (num_rays && !rays) || num_triangles == 0) return -1;
    if ((mode & 1) && num_rays && (!ids || !ts)) return -1;
    if ((mode & 2) && num_rays && !occ) return -1;
    for (uint64_t i = 0; i < 3 * (uint64_t)num_triangles; ++i) {
        if (indices[i] >= num_vertices) return -1;
    }

    Tree tr;
    memset(&tr, 0, sizeof(tr));
    tr.num_tris = num_triangles;
    tr.pos = positions;
    tr.idx = indices;
    tr.margin = hit_margin_of(num_triangles, positions, indices);

    if (!(mode & 4)) {
        tr.nodes = (Node*)malloc(sizeof(Node) * 2 * (size_t)num_triangles);
        tr.prims = (uint32_t*)malloc(sizeof(uint32_t) * num_triangles);
        tr.cent = (double*)malloc(sizeof(double) * 3 * (size_t)num_triangles);
        tr.blo = (double*)malloc(sizeof(double) * 3 * (size_t)num_triangles);
        tr.bhi = (double*)malloc(sizeof(double) * 3 * (size_t)num_triangles);
        double scale = 0.0;
        for (uint32_t i = 0; i < num_triangles; ++i) {
            float const *a, *b, *c;
            tri_verts(&tr, i, &a, &b, &c);
            tr.prims[i] = i;
            for (int k = 0; k < 3; ++k) {
                double lo = a[k], hi = a[k];
                if (b[k] < lo) lo = b[k];
                if (c[k] < lo) lo = c[k];
                if (b[k] > hi) hi = b[k];
                if (c[k] > hi) hi = c[k];
                tr.blo[3 * (size_t)i + k] = lo;
                tr.bhi[3 * (size_t)i + k] = hi;
                tr.cent[3 * (size_t)i + k] = 0.5 * (lo + hi);
                if (fabs(lo) > scale) scale = fabs(lo);
                if (fabs(hi) > scale) scale = fabs(hi);
            }
        }
        tr.pad = ldexp(scale > 0.0 ? scale : 1.0, -14);
        Sort_item* scratch = (Sort_item*)malloc(sizeof(Sort_item) * (size_t)num_triangles);
        build_node(&tr, scratch, 0, num_triangles);
        free(scratch);
    }

    if (num_threads == 0) num_threads = 1;
    if (num_threads > 256) num_threads = 256;
    if ((uint64_t)num_threads > num_rays) num_threads = num_rays ? (uint32_t)num_rays : 1;

    pthread_t th[256];
    Job jobs[256];
    for (uint32_t w = 0; w < num_threads; ++w) {
        jobs[w].tr = &tr;
        jobs[w].rays = rays;
        jobs[w].begin = num_rays * w / num_threads;
        jobs[w].end = num_rays * (w + 1) / num_threads;
        jobs[w].ids = ids;
        jobs[w].ts = ts;
        jobs[w].uvs = uvs;
        jobs[w].occ = occ;
        jobs[w].mode = mode;
        pthread_create(&th[w], 0, run_job, &jobs[w]);
    }
    for (uint32_t w = 0; w < num_threads; ++w) {
        pthread_join(th[w], 0);
    }

    free(tr.nodes);
    free(tr.prims);
    free(tr.cent);
    free(tr.blo);
    free(tr.bhi);
    return 0;
}

/* One Möller-Trumbore evaluation (for classifying disagreements): out = {t, u, v}. */
int32_t oracle_triangle_test(float const* ray, float const* a, float const* b, float const* c,
                             float tmax, float* out) {
    float t, u, v;
    int32_t const pass = mt_test(ray, a, b, c, tmax, &t, &u, &v);
    out[0] = t;
    out[1] = u;
    out[2] = v;
    return pass;
}
