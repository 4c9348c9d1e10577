/*
 * Test infrastructure: an FP64 CPU restatement of the image that sprout_b200's spectral mode
 * (hero-wavelength transport, sprout_b200/csrc/spectral.cuh) estimates, for scenes of
 * participating media, emitters and a uniform environment.  It is the checker of that mode
 * (tests/test_spectral_gpu.py) and nothing in the library calls it.  The reference renders RGB
 * only, so this mode has no reference counterpart: parity is pinned to this restatement.
 *
 * The image is defined by the same ingredients as the GPU's:
 *   - the pinhole camera, the bordered sample grid and the film filter of the RGB renderer
 *     (Perspective::generate_ray, camera_perspective.cpp:47-80; Gaussian radius 1, alpha 1.8,
 *     tabulated over the squared distance at 30 points, filtered.inl:125-187);
 *   - RGB quantities upsampled by the basis S_r, S_g, S_b and read out through the CIE 1931
 *     colour-matching functions (Wyman, Sloan and Shirley 2013) with the round-trip correction
 *     (the formulas of spectral.cuh, restated here in double precision);
 *   - media of density d(x) * (mu_a, mu_s) with a Henyey-Greenstein phase function, density
 *     grids read trilinearly with clamped coordinates (Linear_3D, texture_sampler.cpp:175-283);
 *   - paths cut after max_bounces scattering vertices (no light sample at the last).
 * The estimator is deliberately different from the GPU's: one wavelength per path (uniform),
 * delta tracking against one global majorant with analog albedo weighting, ratio tracking
 * against the same majorant for shadow rays, its own light choice (environment or an emitter
 * by power) with power-heuristic MIS, no Russian roulette, brute-force ray-triangle tests.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define PI 3.14159265358979323846
#define MAX_STEPS 1000000 /* collisions per tracking segment (a closed medium never needs them) */

typedef struct {
    double x, y, z;
} v3;

static v3 V(double x, double y, double z) {
    v3 r = {x, y, z};
    return r;
}
static v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 mul(double s, v3 a) { return V(s * a.x, s * a.y, s * a.z); }
static double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 cross(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static v3 normalize(v3 a) { return mul(1.0 / sqrt(dot(a, a)), a); }

/* splitmix64: one stream per (pixel, sample) */
typedef struct {
    uint64_t s;
} rng_t;
static double uniform(rng_t* r) {
    uint64_t z = (r->s += 0x9E3779B97F4A7C15ull);
    z          = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z          = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

/* ---- colour (spectral.cuh) ---- */
#define LMIN 380.0
#define LMAX 720.0

static double smooth01(double x) {
    x = x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x);
    return x * x * (3.0 - 2.0 * x);
}
static double upsample(double const rgb[3], double l) {
    double const t1 = smooth01((l - 465.0) / 50.0), t2 = smooth01((l - 560.0) / 50.0);
    return rgb[0] * t2 + rgb[1] * (t1 - t2) + rgb[2] * (1.0 - t1);
}
static double lobe(double l, double mu, double a, double b) {
    double const t = (l - mu) / (l < mu ? a : b);
    return exp(-0.5 * t * t);
}
static void response(double l, double out[3]) {
    static double const m[9] = {0.61309732, 0.33952285, 0.04737928, 0.07019422, 0.91635557,
                                0.01345259, 0.02061560, 0.10956983, 0.86981512};
    double const x = 1.056 * lobe(l, 599.8, 37.9, 31.0) + 0.362 * lobe(l, 442.0, 16.0, 26.7) -
                     0.065 * lobe(l, 501.1, 20.4, 26.2);
    double const y = 0.821 * lobe(l, 568.8, 46.9, 40.5) + 0.286 * lobe(l, 530.9, 16.3, 31.1);
    double const z = 1.217 * lobe(l, 437.0, 11.8, 36.0) + 0.681 * lobe(l, 459.0, 26.0, 13.8);
    double const s[3] = {3.2406 * x - 1.5372 * y - 0.4986 * z, -0.9689 * x + 1.8758 * y + 0.0415 * z,
                         0.0557 * x - 0.2040 * y + 1.0570 * z};
    for (int i = 0; i < 3; ++i) {
        out[i] = m[3 * i] * s[0] + m[3 * i + 1] * s[1] + m[3 * i + 2] * s[2];
    }
}
/* C with C G = I, G[i][j] = integral of response_i * basis_j (midpoint rule, 0.25 nm) */
static void readout_matrix(double c[9]) {
    double g[9] = {0};
    for (double l = LMIN + 0.125; l < LMAX; l += 0.25) {
        double r[3];
        response(l, r);
        double const t1 = smooth01((l - 465.0) / 50.0), t2 = smooth01((l - 560.0) / 50.0);
        double const b[3] = {t2, t1 - t2, 1.0 - t1};
        for (int i = 0; i < 3; ++i) {
            for (int j = 0; j < 3; ++j) {
                g[3 * i + j] += r[i] * b[j] * 0.25;
            }
        }
    }
    double const det = g[0] * (g[4] * g[8] - g[5] * g[7]) - g[1] * (g[3] * g[8] - g[5] * g[6]) +
                       g[2] * (g[3] * g[7] - g[4] * g[6]);
    double const id = 1.0 / det;
    c[0] = (g[4] * g[8] - g[5] * g[7]) * id;
    c[1] = (g[2] * g[7] - g[1] * g[8]) * id;
    c[2] = (g[1] * g[5] - g[2] * g[4]) * id;
    c[3] = (g[5] * g[6] - g[3] * g[8]) * id;
    c[4] = (g[0] * g[8] - g[2] * g[6]) * id;
    c[5] = (g[2] * g[3] - g[0] * g[5]) * id;
    c[6] = (g[3] * g[7] - g[4] * g[6]) * id;
    c[7] = (g[1] * g[6] - g[0] * g[7]) * id;
    c[8] = (g[0] * g[4] - g[1] * g[3]) * id;
}

/* ---- scene ---- */
typedef struct {
    uint32_t      num_tris;
    double const* tris;     /* 9 per triangle: a, b, c */
    int32_t const* tri_mat; /* material per triangle */
    int32_t const* mat_type; /* 0 light, 1 medium boundary */
    double const* mat;       /* 8 per material: light: emission rgb, two-sided; medium: mu_a rgb, mu_s rgb,
                                g, uses the grid */
    uint32_t      nx, ny, nz;
    double const* density;   /* z-major, x fastest */
    double const* w2uvw;     /* 12: uvw = M[0..2] . p + M[3], ... */
    double        grid_max;
    double        env[3];
    int32_t       env_light;
    /* lights */
    uint32_t      num_lights;
    uint32_t*     light_tri;
    double*       light_cdf;
    double        light_total;
    double        p_env;
} scene_t;

typedef struct {
    double t;
    int    tri;
} hit_t;

static hit_t closest(scene_t const* s, v3 o, v3 d, double tmin, double tmax) {
    hit_t h = {tmax, -1};
    for (uint32_t i = 0; i < s->num_tris; ++i) {
        double const* t  = s->tris + 9 * (size_t)i;
        v3 const      a  = V(t[0], t[1], t[2]);
        v3 const      e1 = sub(V(t[3], t[4], t[5]), a);
        v3 const      e2 = sub(V(t[6], t[7], t[8]), a);
        v3 const      p  = cross(d, e2);
        double const  det = dot(e1, p);
        if (fabs(det) < 1e-300) {
            continue;
        }
        double const inv = 1.0 / det;
        v3 const     tv  = sub(o, a);
        /* barycentric bounds widened by 1e-9, so that a ray through a shared edge hits one of
           the two triangles (a closed medium boundary has no cracks) */
        double const u   = dot(tv, p) * inv;
        if (u < -1e-9 || u > 1.0 + 1e-9) {
            continue;
        }
        v3 const     q  = cross(tv, e1);
        double const v  = dot(d, q) * inv;
        if (v < -1e-9 || u + v > 1.0 + 1e-9) {
            continue;
        }
        double const tt = dot(e2, q) * inv;
        if (tt > tmin && tt < h.t) {
            h.t   = tt;
            h.tri = (int)i;
        }
    }
    return h;
}

static v3 tri_normal(scene_t const* s, int i) {
    double const* t = s->tris + 9 * (size_t)i;
    return normalize(cross(V(t[3] - t[0], t[4] - t[1], t[5] - t[2]), V(t[6] - t[0], t[7] - t[1], t[8] - t[2])));
}
static double tri_area(scene_t const* s, int i) {
    double const* t = s->tris + 9 * (size_t)i;
    v3 const      c = cross(V(t[3] - t[0], t[4] - t[1], t[5] - t[2]), V(t[6] - t[0], t[7] - t[1], t[8] - t[2]));
    return 0.5 * sqrt(dot(c, c));
}

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

static double density_at(scene_t const* s, v3 p) {
    double const* m = s->w2uvw;
    double uvw[3];
    for (int k = 0; k < 3; ++k) {
        double u = m[4 * k] * p.x + m[4 * k + 1] * p.y + m[4 * k + 2] * p.z + m[4 * k + 3];
        uvw[k]   = u < 0.0 ? 0.0 : (u > 1.0 ? 1.0 : u);
    }
    int const    n[3] = {(int)s->nx, (int)s->ny, (int)s->nz};
    int          lo[3], hi[3];
    double       f[3];
    for (int k = 0; k < 3; ++k) {
        double const x = uvw[k] * n[k] - 0.5;
        double const fl = floor(x);
        f[k]            = x - fl;
        lo[k]           = clampi((int)fl, 0, n[k] - 1);
        hi[k]           = clampi((int)fl + 1, 0, n[k] - 1);
    }
    double acc = 0.0;
    for (int c = 0; c < 8; ++c) {
        int const    x = (c & 1) ? hi[0] : lo[0], y = (c & 2) ? hi[1] : lo[1], z = (c & 4) ? hi[2] : lo[2];
        double const w = ((c & 1) ? f[0] : 1 - f[0]) * ((c & 2) ? f[1] : 1 - f[1]) * ((c & 4) ? f[2] : 1 - f[2]);
        acc += w * s->density[((size_t)z * s->ny + y) * s->nx + x];
    }
    return acc;
}

/* coefficients of medium material m at wavelength l */
static void medium_at(scene_t const* s, int m, double l, double* mu_t, double* mu_s, double* g, int* grid) {
    double const* p = s->mat + 8 * (size_t)m;
    double const  a = upsample(p, l);
    *mu_s           = upsample(p + 3, l);
    *mu_t           = a + *mu_s;
    *g              = p[6];
    *grid           = p[7] != 0.0;
}

/* transmittance along o + t d, t in [0, dist], starting in medium `med` (-1: none) */
static double transmittance(scene_t const* s, v3 o, v3 d, double dist, int med, double l, rng_t* r) {
    double tr = 1.0, t0 = 1e-9;
    for (int crossing = 0; crossing < 64; ++crossing) {
        hit_t const  h   = closest(s, o, d, t0, dist);
        double const end = h.tri >= 0 ? h.t : dist;
        if (med >= 0) {
            double mu_t, mu_s, g;
            int    grid;
            medium_at(s, med, l, &mu_t, &mu_s, &g, &grid);
            if (grid) {
                double const maj = s->grid_max * mu_t;
                if (maj > 0.0) {
                    double t = t0;
                    for (int step = 0; step < MAX_STEPS; ++step) {
                        t -= log(1.0 - uniform(r)) / maj;
                        if (t >= end) {
                            break;
                        }
                        tr *= 1.0 - density_at(s, add(o, mul(t, d))) * mu_t / maj;
                    }
                }
            } else {
                tr *= exp(-mu_t * (end - t0));
            }
        }
        if (h.tri < 0) {
            return tr;
        }
        int const m = s->tri_mat[h.tri];
        if (s->mat_type[m] != 1) {
            return 0.0;
        }
        med = dot(tri_normal(s, h.tri), d) < 0.0 ? m : -1;
        t0  = h.t + 1e-7 * (1.0 + h.t);
    }
    return tr;
}

static double hg(double cos_travel, double g) {
    double const den = 1.0 + g * g - 2.0 * g * cos_travel;
    return (1.0 - g * g) / (4.0 * PI * den * sqrt(den));
}

static void frame(v3 n, v3* t, v3* b) {
    v3 const a = fabs(n.x) > 0.9 ? V(0, 1, 0) : V(1, 0, 0);
    *t         = normalize(cross(a, n));
    *b         = cross(n, *t);
}

/* the light part of the oracle's estimator: its own pdf of sampling direction w at p towards
   an emitter triangle hit at distance dist (or the environment when tri < 0) */
static double light_pdf(scene_t const* s, int tri, double dist, v3 w) {
    if (tri < 0) {
        return s->env_light ? s->p_env / (4.0 * PI) : 0.0;
    }
    for (uint32_t k = 0; k < s->num_lights; ++k) {
        if ((int)s->light_tri[k] == tri) {
            double const prev = k ? s->light_cdf[k - 1] : 0.0;
            double const pick = (1.0 - s->p_env) * (s->light_cdf[k] - prev) / s->light_total;
            double const c    = fabs(dot(tri_normal(s, tri), w));
            return c > 0.0 ? pick * dist * dist / (c * tri_area(s, tri)) : 0.0;
        }
    }
    return 0.0;
}

static double path(scene_t const* s, v3 o, v3 d, double l, uint32_t min_b, uint32_t max_b, rng_t* r) {
    (void)min_b;
    double   L = 0.0, T = 1.0, pdf_prev = 0.0;
    int      med = -1, camera = 1;
    uint32_t depth = 0;
    double   tmin  = 1e-9;
    for (int seg = 0; seg < 4096; ++seg) {
        hit_t const  h     = closest(s, o, d, tmin, 1e300);
        double const t_hit = h.tri >= 0 ? h.t : 1e300;
        int          scattered = 0;
        double       t_sc      = 0.0, g = 0.0;
        if (med >= 0) {
            double mu_t, mu_s;
            int    grid;
            medium_at(s, med, l, &mu_t, &mu_s, &g, &grid);
            double const maj = grid ? s->grid_max * mu_t : mu_t;
            if (maj > 0.0) {
                double t = tmin;
                for (int step = 0; step < MAX_STEPS; ++step) {
                    t -= log(1.0 - uniform(r)) / maj;
                    if (t >= t_hit) {
                        break;
                    }
                    double const real = grid ? density_at(s, add(o, mul(t, d))) * mu_t / maj : 1.0;
                    if (uniform(r) < real) {
                        T *= mu_s / mu_t;
                        t_sc      = t;
                        scattered = 1;
                        break;
                    }
                }
            }
        }
        if (scattered) {
            if (depth >= max_b) {
                break;
            }
            v3 const p = add(o, mul(t_sc, d));
            /* light sample: the environment with probability p_env, else an emitter by power */
            if (s->env_light || s->num_lights) {
                double const u0 = uniform(r), u1 = uniform(r), u2 = uniform(r);
                v3           w;
                double       dist, pdf, Le;
                int          ok = 0;
                if (u0 < s->p_env) {
                    double const z = 1.0 - 2.0 * u1, rad = sqrt(fmax(0.0, 1.0 - z * z)), ph = 2.0 * PI * u2;
                    w    = V(rad * cos(ph), rad * sin(ph), z);
                    dist = 1e300;
                    pdf  = s->p_env / (4.0 * PI);
                    Le   = upsample(s->env, l);
                    ok   = 1;
                } else {
                    double const x  = (u0 - s->p_env) / (1.0 - s->p_env) * s->light_total;
                    uint32_t     k  = 0;
                    while (k + 1 < s->num_lights && s->light_cdf[k] <= x) {
                        ++k;
                    }
                    int const     tri = (int)s->light_tri[k];
                    double const* t   = s->tris + 9 * (size_t)tri;
                    double const  sq  = sqrt(u1);
                    v3 const      a   = V(t[0], t[1], t[2]);
                    v3 const      q   = add(a, add(mul(sq * (1.0 - u2), V(t[3] - t[0], t[4] - t[1], t[5] - t[2])),
                                                mul(sq * u2, V(t[6] - t[0], t[7] - t[1], t[8] - t[2]))));
                    v3 const      ax  = sub(q, p);
                    dist              = sqrt(dot(ax, ax));
                    w                 = mul(1.0 / dist, ax);
                    double const* mp  = s->mat + 8 * (size_t)s->tri_mat[tri];
                    double const  c   = -dot(tri_normal(s, tri), w);
                    if (c > 1e-9 || (mp[3] != 0.0 && c < -1e-9)) {
                        pdf  = light_pdf(s, tri, dist, w);
                        Le   = upsample(mp, l);
                        dist = dist * (1.0 - 1e-7);
                        ok   = pdf > 0.0;
                    }
                }
                if (ok) {
                    double const f = hg(dot(d, w), g);
                    double const wt = pdf * pdf / (pdf * pdf + f * f);
                    double const tr = transmittance(s, p, w, dist, med, l, r);
                    L += T * wt * f * Le * tr / pdf;
                }
            }
            /* phase sample around the travel direction */
            double const x0 = uniform(r), x1 = uniform(r);
            double       ct;
            if (fabs(g) < 1e-3) {
                ct = 1.0 - 2.0 * x0;
            } else {
                double const sq = (1.0 - g * g) / (1.0 - g + 2.0 * g * x0);
                ct              = (1.0 + g * g - sq * sq) / (2.0 * g);
            }
            double const st = sqrt(fmax(0.0, 1.0 - ct * ct)), ph = 2.0 * PI * x1;
            v3           tt, bb;
            frame(d, &tt, &bb);
            d        = add(add(mul(st * cos(ph), tt), mul(st * sin(ph), bb)), mul(ct, d));
            pdf_prev = hg(ct, g);
            o        = p;
            tmin     = 1e-9;
            camera   = 0;
            ++depth;
            continue;
        }
        if (h.tri < 0) {
            if (med < 0 && (camera || s->env_light)) {
                double w = 1.0;
                if (!camera) {
                    double const pl = light_pdf(s, -1, 0.0, d);
                    w               = pdf_prev * pdf_prev / (pdf_prev * pdf_prev + pl * pl);
                }
                L += w * T * upsample(s->env, l);
            }
            break;
        }
        int const    m     = s->tri_mat[h.tri];
        v3 const     n     = tri_normal(s, h.tri);
        double const cos_o = -dot(n, d);
        if (s->mat_type[m] == 0) {
            double const* mp = s->mat + 8 * (size_t)m;
            if (cos_o > 0.0 || mp[3] != 0.0) {
                double w = 1.0;
                if (!camera) {
                    double const pl = light_pdf(s, h.tri, h.t, d);
                    w               = pdf_prev * pdf_prev / (pdf_prev * pdf_prev + pl * pl);
                }
                L += w * T * upsample(mp, l);
            }
            break;
        }
        med  = cos_o > 0.0 ? m : -1;
        tmin = h.t + 1e-7 * (1.0 + h.t);
    }
    return L;
}

/*
 * Renders width x height (linear ACEScg rgb per pixel into out, 3 floats each) with spp samples
 * per bordered pixel; see the file comment for the scene arrays.  Returns 0.
 */
int oracle_spectral_render(uint32_t num_tris, double const* tris, int32_t const* tri_mat, int32_t const* mat_type,
                           double const* mat, uint32_t nx, uint32_t ny, uint32_t nz, double const* density,
                           double const* w2uvw, double const* env, int32_t env_light, uint32_t width, uint32_t height,
                           double fov, double const* rot, double const* pos, uint32_t spp, uint32_t min_bounces,
                           uint32_t max_bounces, uint64_t seed, uint32_t* light_tri, double* light_cdf, double* out,
                           double* weight) {
    scene_t s;
    memset(&s, 0, sizeof(s));
    s.num_tris = num_tris;
    s.tris     = tris;
    s.tri_mat  = tri_mat;
    s.mat_type = mat_type;
    s.mat      = mat;
    s.nx = nx, s.ny = ny, s.nz = nz;
    s.density  = density;
    s.w2uvw    = w2uvw;
    s.grid_max = 0.0;
    for (size_t i = 0; i < (size_t)nx * ny * nz; ++i) {
        s.grid_max = density[i] > s.grid_max ? density[i] : s.grid_max;
    }
    memcpy(s.env, env, sizeof(s.env));
    s.env_light = env_light;
    /* emitters by power: area x largest emission component (two-sided twice) */
    s.light_tri = light_tri;
    s.light_cdf = light_cdf;
    for (uint32_t i = 0; i < num_tris; ++i) {
        int const m = tri_mat[i];
        if (mat_type[m] != 0) {
            continue;
        }
        double const* mp = mat + 8 * (size_t)m;
        double const  e  = fmax(mp[0], fmax(mp[1], mp[2])) * (mp[3] != 0.0 ? 2.0 : 1.0);
        s.light_total += tri_area(&s, (int)i) * e;
        light_tri[s.num_lights] = i;
        light_cdf[s.num_lights] = s.light_total;
        ++s.num_lights;
    }
    s.p_env = env_light ? (s.num_lights ? 0.5 : 1.0) : 0.0;

    double c[9];
    readout_matrix(c);
    double filter[30];
    for (int i = 0; i < 30; ++i) {
        filter[i] = fmax(0.0, exp(-1.8 * (double)i / 29.0) - exp(-1.8));
    }
    memset(out, 0, sizeof(double) * 3 * width * height);
    memset(weight, 0, sizeof(double) * width * height);
    double const ratio = (double)height / width, z = 1.0 / tan(0.5 * fov);
    uint32_t const bw = width + 2, bh = height + 2;
    for (uint32_t pix = 0; pix < bw * bh; ++pix) {
        int const px = (int)(pix % bw) - 1, py = (int)(pix / bw) - 1;
        for (uint32_t k = 0; k < spp; ++k) {
            rng_t r = {seed ^ (((uint64_t)pix << 32) | k) * 0xD1B54A32D192ED03ull};
            double const u = uniform(&r), v = uniform(&r);
            double const cx = px + u, cy = py + v;
            v3           d  = normalize(V(-1.0 + cx * 2.0 / width, ratio - cy * 2.0 * ratio / height, z));
            d               = V(d.x * rot[0] + d.y * rot[3] + d.z * rot[6], d.x * rot[1] + d.y * rot[4] + d.z * rot[7],
                                d.x * rot[2] + d.y * rot[5] + d.z * rot[8]);
            double const l  = LMIN + (LMAX - LMIN) * uniform(&r);
            double const L  = path(&s, V(pos[0], pos[1], pos[2]), d, l, min_bounces, max_bounces, &r);
            double       resp[3], rgb[3];
            response(l, resp);
            for (int i = 0; i < 3; ++i) {
                rgb[i] = (LMAX - LMIN) * L * (c[3 * i] * resp[0] + c[3 * i + 1] * resp[1] + c[3 * i + 2] * resp[2]);
            }
            for (int dy = -1; dy <= 1; ++dy) {
                int const fy = py + dy;
                if (fy < 0 || fy >= (int)height) {
                    continue;
                }
                for (int dx = -1; dx <= 1; ++dx) {
                    int const fx = px + dx;
                    if (fx < 0 || fx >= (int)width) {
                        continue;
                    }
                    double wt = 1.0;
                    double const offs[2] = {u - 0.5 - dx, v - 0.5 - dy};
                    for (int a = 0; a < 2; ++a) {
                        double const x = fmin(offs[a] * offs[a], 1.0) * 29.0;
                        int const    o = (int)x;
                        int const    o1 = o + 1 < 30 ? o + 1 : 29;
                        wt *= filter[o] + (x - o) * (filter[o1] - filter[o]);
                    }
                    size_t const q = (size_t)fy * width + fx;
                    for (int i = 0; i < 3; ++i) {
                        out[3 * q + i] += wt * rgb[i];
                    }
                    weight[q] += wt;
                }
            }
        }
    }
    for (size_t q = 0; q < (size_t)width * height; ++q) {
        double const iw = weight[q] > 0.0 ? 1.0 / weight[q] : 0.0;
        for (int i = 0; i < 3; ++i) {
            out[3 * q + i] *= iw;
        }
    }
    return 0;
}
