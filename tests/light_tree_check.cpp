// Structural check of the host light-tree build (sprout_b200/csrc/light_tree.cpp), compiled and
// run by tests/test_light_tree.py.  Builds trees over seeded random emitters (clustered,
// flat, two-sided, degenerate) and checks every invariant the device walk relies on:
//   - every light appears exactly once in tree order, and order[] inverts the mapping;
//   - inner nodes' children are adjacent, leaves hold 1..4 lights, the lights of a subtree are
//     a contiguous range split at `middle`;
//   - node power is the sum of its lights' powers, node variance their population variance
//     (and variance + mean^2) and node light count their number;
//   - a splitting walk returns at most Max_light_picks lights (max_split_picks);
//   - a node's bounding sphere contains its lights' triangles and its cone contains their
//     normals (cos spread -1 when a two-sided light is below);
//   - an emitting medium's light (a box, Light_input::volume != 0) is stored as
//     (centre, -volume) with cone spread -1, a triangle with its (non-negative) area.
// Prints "ok <name> <nodes> <depth> <most picks>" per tree or the first violation, and exits
// non-zero on failure.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "../sprout_b200/csrc/light_tree.hpp"

using spb::render::Light_input;
using spb::render::Light_tree;

namespace {

uint32_t u32(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

struct Checker {
    Light_tree const&               t;
    std::vector<Light_input> const& in;
    std::vector<int>                seen;
    std::vector<uint32_t>           by_tri;  // triangle id -> input index
    bool                            ok = true;

    void fail(char const* what, uint32_t node) {
        if (ok) {
            std::printf("FAIL %s at node %u\n", what, node);
        }
        ok = false;
    }

    float const* node(uint32_t n) const { return &t.nodes[spb::render::Light_node_floats * size_t(n)]; }

    // light (tree order) -> input (its stored material is 2 * slot + 5)
    Light_input const& light(uint32_t o) const {
        return in[by_tri[(u32(t.tris[12 * size_t(o) + 11]) - 5u) / 2u]];
    }

    // returns the [begin, end) range of lights of the subtree, checks contents
    void walk(uint32_t n, uint32_t& begin, uint32_t& end, double& power, int depth) {
        double power2 = 0.0;
        walk(n, begin, end, power, power2, depth);
    }
    void walk(uint32_t n, uint32_t& begin, uint32_t& end, double& power, double& power2, int depth) {
        if (depth > 64) {
            fail("depth", n);
            return;
        }
        float const*   nd    = node(n);
        uint32_t const first = u32(nd[9]);
        uint32_t const count = u32(nd[10]);
        if (count != 0) {
            if (count > spb::render::Light_leaf_size || first + count > t.num_lights) {
                fail("leaf range", n);
                return;
            }
            begin  = first;
            end    = first + count;
            power  = 0.0;
            power2 = 0.0;
            for (uint32_t o = first; o < end; ++o) {
                ++seen[o];
                double const p = t.cones[12 * size_t(o) + 8];
                power += p;
                power2 += p * p;
            }
        } else {
            if (first + 1 >= t.num_nodes) {
                fail("child index", n);
                return;
            }
            uint32_t b0, e0, b1, e1;
            double   p0, p1, q0, q1;
            walk(first, b0, e0, p0, q0, depth + 1);
            walk(first + 1, b1, e1, p1, q1, depth + 1);
            if (e0 != b1 || u32(nd[11]) != b1) {
                fail("middle", n);
            }
            begin  = b0;
            end    = e1;
            power  = p0 + p1;
            power2 = q0 + q1;
        }
        if (std::fabs(power - nd[8]) > 1e-4 * std::fabs(power) + 1e-6) {
            fail("power", n);
        }
        uint32_t const lights = end - begin;
        if (u32(nd[13]) != lights) {
            fail("light count", n);
        }
        double const mean     = power / lights;
        double const variance = std::fabs(power2 / lights - mean * mean);
        if (std::fabs(variance - nd[12]) > 1e-3 * variance + 1e-3 * mean * mean + 1e-9 ||
            std::fabs(variance + mean * mean - nd[14]) > 1e-4 * (variance + mean * mean) + 1e-9) {
            fail("variance", n);
        }
        // bounds of every light below
        double const c[3] = {nd[0], nd[1], nd[2]};
        double const r    = nd[3];
        double const ax[3] = {nd[4], nd[5], nd[6]};
        double const cos_o = nd[7];
        for (uint32_t o = begin; o < end; ++o) {
            Light_input const& l = light(o);
            for (double const* v : {l.a, l.b, l.c}) {
                double const d = std::sqrt((v[0] - c[0]) * (v[0] - c[0]) + (v[1] - c[1]) * (v[1] - c[1]) +
                                           (v[2] - c[2]) * (v[2] - c[2]));
                if (d > r * (1.0 + 1e-5) + 1e-6) {
                    fail("sphere", n);
                }
            }
            float const* lc = &t.cones[12 * size_t(o)];
            if (lc[7] < 0.f) {
                if (cos_o > -1.0) {
                    fail("two-sided cone", n);
                }
            } else if (cos_o > -1.0) {
                double const cd = ax[0] * lc[4] + ax[1] * lc[5] + ax[2] * lc[6];
                if (cd < cos_o - 1e-4) {
                    fail("cone", n);
                }
            }
        }
    }
};

bool check(std::vector<Light_input> const& in, uint32_t num_triangles, char const* name) {
    Light_tree t;
    spb::render::build_light_tree(in, num_triangles, t);
    if (t.num_lights != in.size()) {
        std::printf("FAIL %s: %u lights in tree, %zu given\n", name, t.num_lights, in.size());
        return false;
    }
    Checker k{t, in, std::vector<int>(in.size(), 0), std::vector<uint32_t>(num_triangles, 0)};
    for (size_t i = 0; i < in.size(); ++i) {
        k.by_tri[in[i].slot] = uint32_t(i);
    }
    uint32_t b, e;
    double   p;
    k.walk(0, b, e, p, 0);
    if (k.ok && (b != 0 || e != t.num_lights)) {
        k.fail("root range", 0);
    }
    for (size_t o = 0; k.ok && o < in.size(); ++o) {
        if (k.seen[o] != 1) {
            k.fail("light seen once", uint32_t(o));
        }
        // the light at tree position o carries its material; its slot maps back to o
        uint32_t const material = u32(t.tris[12 * o + 11]);
        uint32_t const slot     = (material - 5u) / 2u;
        if (material != 2u * slot + 5u || slot >= num_triangles || t.order[slot] != o) {
            k.fail("order", uint32_t(o));
            break;
        }
        Light_input const& li = in[k.by_tri[slot]];
        float const        w  = t.tris[12 * o + 3];
        if (li.volume != 0 ? (w != -float(li.volume) || t.cones[12 * o + 7] != -1.f) : !(w >= 0.f)) {
            k.fail("volume or triangle entry", uint32_t(o));
        }
    }
    uint32_t const picks = spb::render::max_split_picks(t, 0);
    if (k.ok && (picks == 0 || picks > spb::render::Max_light_picks ||
                 spb::render::max_split_picks(t, spb::render::Max_split_depth) != 1u ||
                 (in.size() <= spb::render::Light_leaf_size && picks != in.size()))) {
        std::printf("FAIL %s: max_split_picks %u\n", name, picks);
        k.ok = false;
    }
    if (k.ok) {
        std::printf("ok %s %u %u %u\n", name, t.num_nodes, t.depth, picks);
    }
    return k.ok;
}

std::vector<Light_input> emitters(int n, int kind, uint32_t seed) {
    std::mt19937                           g(seed);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    std::vector<Light_input>               v;
    for (int i = 0; i < n; ++i) {
        Light_input l;
        double      c[3] = {u(g) * 10.0, u(g) * 10.0, kind == 1 ? 2.0 : u(g) * 10.0};
        if (kind == 2) {  // two clusters far apart
            c[0] = (i & 1) ? 100.0 + u(g) : u(g);
        }
        for (int k = 0; k < 3; ++k) {
            double const s = kind == 3 ? 0.0 : 0.1;  // kind 3: zero-extent points
            l.a[k]         = c[k] + s * (u(g) - 0.5);
            l.b[k]         = c[k] + s * (u(g) - 0.5);
            l.c[k]         = c[k] + s * (u(g) - 0.5);
        }
        if (kind == 1) {
            l.a[2] = l.b[2] = l.c[2] = 2.0;  // coplanar, identical normals
        }
        if (kind == 4 && i % 5 == 2) {  // an emitting medium's box among the triangles
            for (int k = 0; k < 3; ++k) {
                l.a[k] = c[k] - 0.3;
                l.b[k] = c[k] + 0.3;
                l.c[k] = c[k];
            }
            l.volume = uint32_t(i / 5) + 1;
        }
        l.power     = std::exp(4.0 * u(g));
        l.two_sided = (i % 7) == 3 || l.volume != 0;
        l.slot      = uint32_t(3 * i + 1);
        l.material  = 2u * l.slot + 5u;
        v.push_back(l);
    }
    return v;
}

}  // namespace

int main() {
    bool ok = true;
    ok &= check(emitters(1, 0, 1), 4, "single");
    ok &= check(emitters(5, 0, 2), 16, "five");
    ok &= check(emitters(4096, 0, 3), 3 * 4096 + 2, "random4096");
    ok &= check(emitters(1000, 1, 4), 3 * 1000 + 2, "coplanar");
    ok &= check(emitters(999, 2, 5), 3 * 999 + 2, "clusters");
    ok &= check(emitters(300, 3, 6), 3 * 300 + 2, "points");
    ok &= check(emitters(500, 4, 7), 3 * 500 + 2, "volumes");
    return ok ? 0 : 1;
}
