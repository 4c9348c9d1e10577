/*
 * CPU restatement of the cast benchmark's synthetic inputs.
 * TEST INFRASTRUCTURE ONLY: the bench's reference arm makes its mesh and rays with it, so
 * that timing the reference's own traversal loads nothing of the product library; a CPU test
 * checks that it reproduces the product's spb_synth_sphere_mesh / spb_synth_rays bit for bit.
 *
 * The inputs (no counterpart in the reference, which has no benchmark scenes):
 *   - mesh: a tetrahedron with faces subdivided n x n, lattice points projected to the unit
 *     sphere and displaced radially by amplitude * fBm (6 octaves of 3-D gradient noise,
 *     lacunarity 2, gain 0.5, base frequency 3, octave offsets 17 * (1, 0.5, 0.25) * o,
 *     normalised by the summed octave weights; a seeded permutation of 0..255 and the 12
 *     cube-edge gradients, quintic fade), all in double precision; vertices numbered in order
 *     of first use when the faces are walked row by row;
 *   - rays: PCG32 (O'Neill, XSH-RR) seeded as the reference's rnd::Generator::start
 *     (source/base/random/generator.inl:16-24) with sequence = ray index; origin uniform in
 *     [-extent, extent]^3, z = 1 - 2u, azimuth from a point rejection-sampled in the unit disk,
 *     min_t 0, max_t = scene::Ray_max_t (source/core/scene/scene_constants.hpp:10).
 *
 * Build: compiled into libcast_oracle.so beside cast_oracle.c (gcc -O2 -ffp-contract=off).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    uint64_t state;
    uint64_t inc;
} Pcg;

static uint32_t pcg_next(Pcg* g) {
    uint64_t const old = g->state;
    g->state           = old * 6364136223846793005ull + (g->inc | 1u);
    uint32_t const x   = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t const rot = (uint32_t)(old >> 59u);
    return (x >> rot) | (x << ((0u - rot) & 31u));
}

static void pcg_start(Pcg* g, uint64_t seed, uint64_t sequence) {
    g->state = 0;
    g->inc   = (sequence << 1u) | 1u;
    pcg_next(g);
    g->state += seed;
    pcg_next(g);
}

static float pcg_uniform(Pcg* g) {
    uint32_t const bits = (pcg_next(g) & 0x007FFFFFu) | 0x3F800000u;
    float          f;
    memcpy(&f, &bits, 4);
    return f - 1.f;
}

typedef struct {
    uint8_t p[256];
} Perm;

static void perm_init(Perm* pm, uint32_t seed) {
    for (uint32_t i = 0; i < 256; ++i) {
        pm->p[i] = (uint8_t)i;
    }
    Pcg g;
    pcg_start(&g, seed, 0x5eed);
    for (uint32_t i = 255; i > 0; --i) {
        uint32_t const j = pcg_next(&g) % (i + 1);
        uint8_t const  t = pm->p[i];
        pm->p[i]         = pm->p[j];
        pm->p[j]         = t;
    }
}

static double fade(double t) { return t * t * t * (t * (t * 6. - 15.) + 10.); }

static double lerp(double a, double b, double t) { return a + t * (b - a); }

static double grad(uint32_t h, double x, double y, double z) {
    switch (h % 12) {
        case 0: return x + y;
        case 1: return -x + y;
        case 2: return x - y;
        case 3: return -x - y;
        case 4: return x + z;
        case 5: return -x + z;
        case 6: return x - z;
        case 7: return -x - z;
        case 8: return y + z;
        case 9: return -y + z;
        case 10: return y - z;
        default: return -y - z;
    }
}

static double noise3(Perm const* pm, double x, double y, double z) {
    double const fx = floor(x), fy = floor(y), fz = floor(z);
    int32_t const ix = (int32_t)fx & 255, iy = (int32_t)fy & 255, iz = (int32_t)fz & 255;
    double const  rx = x - fx, ry = y - fy, rz = z - fz;
    double        c[8];
    for (int32_t k = 0; k < 8; ++k) {
        int32_t const  dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
        uint32_t const h  = pm->p[(pm->p[(pm->p[(ix + dx) & 255] + (iy + dy)) & 255] + (iz + dz)) & 255];
        c[k]              = grad(h, rx - dx, ry - dy, rz - dz);
    }
    double const u = fade(rx), v = fade(ry), w = fade(rz);
    double const y0 = lerp(lerp(c[0], c[1], u), lerp(c[2], c[3], u), v);
    double const y1 = lerp(lerp(c[4], c[5], u), lerp(c[6], c[7], u), v);
    return lerp(y0, y1, w);
}

static double fbm6(Perm const* pm, double x, double y, double z) {
    double sum = 0., norm = 0., amp = 1., freq = 3.;
    for (int32_t o = 0; o < 6; ++o) {
        double const off = 17.0 * (double)o;
        sum += amp * noise3(pm, x * freq + off, y * freq + 0.5 * off, z * freq + 0.25 * off);
        norm += amp;
        amp *= 0.5;
        freq *= 2.;
    }
    return sum / norm;
}

/* Open-addressing map from a lattice point's corner weights to its vertex id. */
typedef struct {
    uint64_t* keys;
    uint32_t* vals;
    uint64_t  mask;
} Map;

static uint64_t mix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    return k;
}

typedef struct {
    Map          map;
    Perm         perm;
    float        amplitude;
    float*       positions;
    uint32_t     next;
} Mesh_state;

static uint32_t lattice_vertex(Mesh_state* m, uint32_t const w[4]) {
    static double const corners[4][3] = {{1., 1., 1.}, {1., -1., -1.}, {-1., 1., -1.}, {-1., -1., 1.}};
    uint64_t const key = (uint64_t)w[0] | ((uint64_t)w[1] << 16) | ((uint64_t)w[2] << 32) | ((uint64_t)w[3] << 48);
    uint64_t       h   = mix64(key) & m->map.mask;
    while (m->map.keys[h] != UINT64_MAX) {
        if (m->map.keys[h] == key) {
            return m->map.vals[h];
        }
        h = (h + 1) & m->map.mask;
    }
    double p[3] = {0., 0., 0.};
    for (int32_t k = 0; k < 4; ++k) {
        for (int32_t a = 0; a < 3; ++a) {
            p[a] += (double)w[k] * corners[k][a];
        }
    }
    double const len = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    double const ux = p[0] / len, uy = p[1] / len, uz = p[2] / len;
    double const r  = 1. + (double)m->amplitude * fbm6(&m->perm, ux, uy, uz);
    uint32_t const id = m->next++;
    m->positions[3 * id + 0] = (float)(ux * r);
    m->positions[3 * id + 1] = (float)(uy * r);
    m->positions[3 * id + 2] = (float)(uz * r);
    m->map.keys[h] = key;
    m->map.vals[h] = id;
    return id;
}

/* positions: (2 n^2 + 2) x 3 floats; indices: 4 n^2 x 3.  Returns 0 on success. */
int32_t oracle_synth_sphere_mesh(uint32_t n, float amplitude, uint32_t seed, float* positions,
                                 uint32_t* indices) {
    static uint32_t const faces[4][3] = {{0, 2, 1}, {0, 1, 3}, {0, 3, 2}, {1, 2, 3}};
    if (n == 0 || n > 16384 || !positions || !indices) {
        return -1;
    }
    uint64_t const nv  = 2ull * n * n + 2;
    uint64_t       cap = 1;
    while (cap < 2 * nv) {
        cap <<= 1;
    }
    Mesh_state m;
    m.map.keys  = (uint64_t*)malloc(cap * sizeof(uint64_t));
    m.map.vals  = (uint32_t*)malloc(cap * sizeof(uint32_t));
    m.map.mask  = cap - 1;
    m.amplitude = amplitude;
    m.positions = positions;
    m.next      = 0;
    if (!m.map.keys || !m.map.vals) {
        free(m.map.keys);
        free(m.map.vals);
        return -1;
    }
    memset(m.map.keys, 0xFF, cap * sizeof(uint64_t));
    perm_init(&m.perm, seed);
    uint64_t tri = 0;
    for (int f = 0; f < 4; ++f) {
        for (uint32_t i = 0; i < n; ++i) {
            for (uint32_t j = 0; i + j < n; ++j) {
                uint32_t w[4];
                uint32_t v[4];
                uint32_t const di[4] = {0, 1, 0, 1};
                uint32_t const dj[4] = {0, 0, 1, 1};
                int const      corners_needed = (i + j + 1 < n) ? 4 : 3;
                for (int c = 0; c < corners_needed; ++c) {
                    memset(w, 0, sizeof(w));
                    uint32_t const ii = i + di[c], jj = j + dj[c];
                    w[faces[f][0]] += n - ii - jj;
                    w[faces[f][1]] += ii;
                    w[faces[f][2]] += jj;
                    v[c] = lattice_vertex(&m, w);
                }
                indices[3 * tri + 0] = v[0];
                indices[3 * tri + 1] = v[1];
                indices[3 * tri + 2] = v[2];
                ++tri;
                if (corners_needed == 4) {
                    indices[3 * tri + 0] = v[1];
                    indices[3 * tri + 1] = v[3];
                    indices[3 * tri + 2] = v[2];
                    ++tri;
                }
            }
        }
    }
    free(m.map.keys);
    free(m.map.vals);
    return (tri == 4ull * n * n && m.next == nv) ? 0 : -1;
}

typedef struct {
    uint64_t first, begin, end;
    uint32_t seed;
    float    extent;
    float*   rays;
} Ray_job;

static void* ray_job(void* arg) {
    Ray_job const* j = (Ray_job const*)arg;
    float const ray_max_t = 3.4027715434167032e+38f;
    for (uint64_t k = j->begin; k < j->end; ++k) {
        Pcg g;
        pcg_start(&g, j->seed, j->first + k);
        float* r = j->rays + 8 * k;
        for (int a = 0; a < 3; ++a) {
            r[a] = j->extent * (2.f * pcg_uniform(&g) - 1.f);
        }
        r[3] = 0.f;
        float const z = 1.f - 2.f * pcg_uniform(&g);
        float       a, b, s;
        do {
            a = 2.f * pcg_uniform(&g) - 1.f;
            b = 2.f * pcg_uniform(&g) - 1.f;
            s = a * a + b * b;
        } while (s > 1.f || s < 1e-12f);
        float const one_minus = 1.f - z * z;
        float const rr        = sqrtf(one_minus > 0.f ? one_minus : 0.f);
        float const k2        = rr / sqrtf(s);
        r[4] = a * k2;
        r[5] = b * k2;
        r[6] = z;
        r[7] = ray_max_t;
    }
    return 0;
}

/* rays: count x 8 floats, ray k drawn from stream (seed, first + k). */
int32_t oracle_synth_rays(uint64_t first, uint64_t count, uint32_t seed, float extent, float* rays,
                          uint32_t threads) {
    if (count > 0 && !rays) {
        return -1;
    }
    if (threads == 0) {
        threads = 1;
    }
    if (threads > 256) {
        threads = 256;
    }
    pthread_t th[256];
    Ray_job   jobs[256];
    uint64_t const per = (count + threads - 1) / threads;
    uint32_t       used = 0;
    for (uint32_t w = 0; w < threads; ++w) {
        uint64_t const b = (uint64_t)w * per;
        if (b >= count) {
            break;
        }
        jobs[w] = (Ray_job){first, b, b + per < count ? b + per : count, seed, extent, rays};
        pthread_create(&th[w], 0, ray_job, &jobs[w]);
        ++used;
    }
    for (uint32_t w = 0; w < used; ++w) {
        pthread_join(th[w], 0);
    }
    return 0;
}
