// Host build of the light tree (light_tree.hpp).  The reference's builder
// (scene/light/light_tree_builder.cpp:436-760) splits by a binned cost over power, bounds and
// cone; this one evaluates the surface-area-orientation heuristic of Estevez and Kulla (2018)
// over 12 centroid bins per axis, in double precision.
#include "light_tree.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <numeric>

namespace spb::render {

namespace {

constexpr double Pi       = 3.14159265358979323846;
constexpr int    Num_bins = 12;

struct Box {
    double lo[3] = {1e300, 1e300, 1e300};
    double hi[3] = {-1e300, -1e300, -1e300};

    void add(double const p[3]) {
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], p[k]);
            hi[k] = std::max(hi[k], p[k]);
        }
    }
    void add(Box const& b) {
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], b.lo[k]);
            hi[k] = std::max(hi[k], b.hi[k]);
        }
    }
    bool   empty() const { return lo[0] > hi[0]; }
    double extent(int k) const { return empty() ? 0.0 : hi[k] - lo[k]; }
    double area() const {
        double const x = extent(0), y = extent(1), z = extent(2);
        return 2.0 * (x * y + y * z + z * x);
    }
};

// Cone of emitter normals: axis and spread angle theta_o in [0, pi]; theta_o < 0 marks the
// empty cone.  Emitters are triangles, so the emission spread around each normal is pi / 2.
struct Cone {
    double axis[3] = {0.0, 0.0, 1.0};
    double theta   = -1.0;
};

double dot(double const a[3], double const b[3]) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// Smallest cone containing both (Estevez and Kulla 2018, Listing 1).
Cone merge(Cone a, Cone b) {
    if (a.theta < 0.0) {
        return b;
    }
    if (b.theta < 0.0) {
        return a;
    }
    if (b.theta > a.theta) {
        std::swap(a, b);
    }
    double const theta_d = std::acos(std::clamp(dot(a.axis, b.axis), -1.0, 1.0));
    if (std::min(theta_d + b.theta, Pi) <= a.theta) {
        return a;
    }
    double const o = 0.5 * (a.theta + theta_d + b.theta);
    if (o >= Pi) {
        a.theta = Pi;
        return a;
    }
    double const rot = o - a.theta;
    // rotate a.axis towards b.axis by rot inside their common plane
    double const c = dot(a.axis, b.axis);
    double       perp[3];
    for (int k = 0; k < 3; ++k) {
        perp[k] = b.axis[k] - c * a.axis[k];
    }
    double const pl = std::sqrt(dot(perp, perp));
    Cone         r;
    r.theta = o;
    if (pl < 1e-12) {
        // (anti)parallel axes: no rotation plane; bound conservatively by the whole sphere
        std::memcpy(r.axis, a.axis, sizeof(r.axis));
        r.theta = c > 0.0 ? a.theta : Pi;
        return r;
    }
    double const cr = std::cos(rot), sr = std::sin(rot);
    double       len = 0.0;
    for (int k = 0; k < 3; ++k) {
        r.axis[k] = cr * a.axis[k] + sr * perp[k] / pl;
        len += r.axis[k] * r.axis[k];
    }
    len = std::sqrt(len);
    for (double& v : r.axis) {
        v /= len;
    }
    return r;
}

// Orientation measure M_Omega of a cone with emission spread pi / 2 (Estevez and Kulla 2018,
// eq. 1).
double orientation_measure(Cone const& c) {
    if (c.theta < 0.0) {
        return 0.0;
    }
    double const to = c.theta;
    double const tw = std::min(to + 0.5 * Pi, Pi);
    double const so = std::sin(to), co = std::cos(to);
    return 2.0 * Pi * (1.0 - co) +
           0.5 * Pi * (2.0 * tw * so - std::cos(to - 2.0 * tw) - 2.0 * to * so + co);
}

struct Item {
    Box    box;
    double centroid[3];
    Cone   cone;
    double power;
    double area;
    bool   two_sided;
};

struct Bin {
    Box    box;
    Cone   cone;
    double power = 0.0;
    double power2 = 0.0;  // sum of squared powers (for the node's variance)
    int    count = 0;

    void add(Item const& it) {
        box.add(it.box);
        cone = merge(cone, it.cone);
        power += it.power;
        power2 += it.power * it.power;
        ++count;
    }
    void add(Bin const& b) {
        box.add(b.box);
        cone = merge(cone, b.cone);
        power += b.power;
        power2 += b.power2;
        count += b.count;
    }
    // Population variance of the powers (every light here has a positive power).
    double variance() const {
        if (count == 0) {
            return 0.0;
        }
        double const mean = power / count;
        return std::fabs(power2 / count - mean * mean);
    }
    double cost() const { return count ? power * box.area() * orientation_measure(cone) : 0.0; }
};

struct Builder {
    std::vector<Item> const& items;
    std::vector<uint32_t>&   index;
    Light_tree&              out;

    void put_float4(std::vector<float>& v, double x, double y, double z, double w) {
        v.push_back(float(x));
        v.push_back(float(y));
        v.push_back(float(z));
        v.push_back(float(w));
    }

    static float bits(uint32_t u) {
        float f;
        std::memcpy(&f, &u, 4);
        return f;
    }

    void write_node(uint32_t node, Bin const& b, uint32_t first, uint32_t count, uint32_t middle) {
        float* n = &out.nodes[Light_node_floats * size_t(node)];
        double c[3], r2 = 0.0;
        for (int k = 0; k < 3; ++k) {
            c[k] = 0.5 * (b.box.lo[k] + b.box.hi[k]);
            r2 += 0.25 * b.box.extent(k) * b.box.extent(k);
        }
        n[0]  = float(c[0]);
        n[1]  = float(c[1]);
        n[2]  = float(c[2]);
        n[3]  = float(std::sqrt(r2));
        n[4]  = float(b.cone.axis[0]);
        n[5]  = float(b.cone.axis[1]);
        n[6]  = float(b.cone.axis[2]);
        n[7]  = float(b.cone.theta >= Pi ? -1.0 : std::cos(b.cone.theta));
        n[8]  = float(b.power);
        n[9]  = bits(first);
        n[10] = bits(count);
        n[11] = bits(middle);
        double const mean = b.count ? b.power / b.count : 0.0;
        n[12] = float(b.variance());
        n[13] = bits(uint32_t(b.count));
        n[14] = float(b.variance() + mean * mean);
        n[15] = 0.f;
    }

    // Builds the subtree of index[begin, end) into node; returns its depth.
    uint32_t build(uint32_t node, uint32_t begin, uint32_t end) {
        Bin all;
        Box cbox;
        for (uint32_t i = begin; i < end; ++i) {
            all.add(items[index[i]]);
            cbox.add(items[index[i]].centroid);
        }
        uint32_t const n = end - begin;
        if (n <= Light_leaf_size) {
            write_node(node, all, begin, n, 0);
            return 1;
        }
        double max_extent = 0.0;
        for (int k = 0; k < 3; ++k) {
            max_extent = std::max(max_extent, all.box.extent(k));
        }
        double best      = 1e300;
        int    best_axis = -1;
        int    best_bin  = 0;
        for (int axis = 0; axis < 3; ++axis) {
            double const ext = cbox.extent(axis);
            if (!(ext > 0.0)) {
                continue;
            }
            std::array<Bin, Num_bins> bins;
            for (uint32_t i = begin; i < end; ++i) {
                Item const& it = items[index[i]];
                int const   b  = std::min(Num_bins - 1,
                                          int(Num_bins * (it.centroid[axis] - cbox.lo[axis]) / ext));
                bins[b].add(it);
            }
            std::array<Bin, Num_bins> right;
            Bin                       acc;
            for (int b = Num_bins - 1; b > 0; --b) {
                acc.add(bins[b]);
                right[b] = acc;
            }
            // Elongated boxes: regularise by the ratio of the longest extent to this axis'.
            double const kr = max_extent / std::max(all.box.extent(axis), 1e-300);
            Bin          left;
            for (int b = 1; b < Num_bins; ++b) {
                left.add(bins[b - 1]);
                if (left.count == 0 || right[b].count == 0) {
                    continue;
                }
                double const cost = kr * (left.cost() + right[b].cost());
                if (cost < best) {
                    best      = cost;
                    best_axis = axis;
                    best_bin  = b;
                }
            }
        }
        uint32_t mid = begin + n / 2;
        if (best_axis >= 0) {
            double const ext = cbox.extent(best_axis);
            auto const   it  = std::partition(
                index.begin() + begin, index.begin() + end, [&](uint32_t l) {
                    int const b = std::min(
                        Num_bins - 1,
                        int(Num_bins * (items[l].centroid[best_axis] - cbox.lo[best_axis]) / ext));
                    return b < best_bin;
                });
            mid = uint32_t(it - index.begin());
        }
        if (mid == begin || mid == end) {
            // every centroid in one bin: median split on the widest centroid axis
            int axis = 0;
            for (int k = 1; k < 3; ++k) {
                if (cbox.extent(k) > cbox.extent(axis)) {
                    axis = k;
                }
            }
            mid = begin + n / 2;
            std::nth_element(index.begin() + begin, index.begin() + mid, index.begin() + end,
                             [&](uint32_t x, uint32_t y) {
                                 return items[x].centroid[axis] < items[y].centroid[axis];
                             });
        }
        uint32_t const child = out.num_nodes;
        out.num_nodes += 2;
        out.nodes.resize(Light_node_floats * size_t(out.num_nodes));
        write_node(node, all, child, 0, mid);
        uint32_t const d0 = build(child, begin, mid);
        uint32_t const d1 = build(child + 1, mid, end);
        return 1 + std::max(d0, d1);
    }
};

}  // namespace

void build_light_tree(std::vector<Light_input> const& lights, uint32_t num_slots,
                      Light_tree& out) {
    out = Light_tree();
    out.order.assign(num_slots, 0xFFFFFFFFu);
    if (lights.empty()) {
        return;
    }
    std::vector<Item> items(lights.size());
    for (size_t l = 0; l < lights.size(); ++l) {
        Light_input const& in = lights[l];
        Item&              it = items[l];
        it.box.add(in.a);
        it.box.add(in.b);
        it.box.add(in.c);
        if (in.volume != 0) {
            // an emitting medium: its box, radiating in every direction
            for (int k = 0; k < 3; ++k) {
                it.centroid[k]  = 0.5 * (in.a[k] + in.b[k]);
                it.cone.axis[k] = k == 2 ? 1.0 : 0.0;
            }
            it.cone.theta = Pi;
            it.power      = in.power;
            it.area       = 0.0;
            it.two_sided  = true;
            continue;
        }
        double e1[3], e2[3], n[3];
        for (int k = 0; k < 3; ++k) {
            it.centroid[k] = (in.a[k] + in.b[k] + in.c[k]) / 3.0;
            e1[k]          = in.b[k] - in.a[k];
            e2[k]          = in.c[k] - in.a[k];
        }
        n[0] = e1[1] * e2[2] - e1[2] * e2[1];
        n[1] = e1[2] * e2[0] - e1[0] * e2[2];
        n[2] = e1[0] * e2[1] - e1[1] * e2[0];
        double const len = std::sqrt(dot(n, n));
        for (int k = 0; k < 3; ++k) {
            it.cone.axis[k] = len > 0.0 ? n[k] / len : (k == 2 ? 1.0 : 0.0);
        }
        it.cone.theta = in.two_sided ? Pi : 0.0;
        it.power      = in.power;
        it.area       = 0.5 * len;
        it.two_sided  = in.two_sided;
    }
    std::vector<uint32_t> index(lights.size());
    std::iota(index.begin(), index.end(), 0u);
    out.num_nodes = 1;
    out.nodes.resize(Light_node_floats);
    Builder b{items, index, out};
    out.depth      = b.build(0, 0, uint32_t(lights.size()));
    out.num_lights = uint32_t(lights.size());
    out.cones.reserve(12 * lights.size());
    out.tris.reserve(12 * lights.size());
    for (uint32_t o = 0; o < out.num_lights; ++o) {
        uint32_t const     l  = index[o];
        Item const&        it = items[l];
        Light_input const& in = lights[l];
        double             c[3], r2 = 0.0;
        for (int k = 0; k < 3; ++k) {
            c[k] = 0.5 * (it.box.lo[k] + it.box.hi[k]);
            r2 += 0.25 * it.box.extent(k) * it.box.extent(k);
        }
        b.put_float4(out.cones, c[0], c[1], c[2], std::sqrt(r2));
        b.put_float4(out.cones, it.cone.axis[0], it.cone.axis[1], it.cone.axis[2],
                     it.two_sided ? -1.0 : 1.0);
        b.put_float4(out.cones, it.power, 0.0, 0.0, 0.0);
        if (in.volume != 0) {
            b.put_float4(out.tris, c[0], c[1], c[2], -double(in.volume));
            b.put_float4(out.tris, 0.0, 0.0, 0.0, 0.0);
            b.put_float4(out.tris, 0.0, 0.0, 0.0, 0.0);
            out.tris.back()    = Builder::bits(in.material);
            out.order[in.slot] = o;
            continue;
        }
        b.put_float4(out.tris, in.a[0], in.a[1], in.a[2], it.area);
        b.put_float4(out.tris, in.b[0] - in.a[0], in.b[1] - in.a[1], in.b[2] - in.a[2], 0.0);
        b.put_float4(out.tris, in.c[0] - in.a[0], in.c[1] - in.a[1], in.c[2] - in.a[2], 0.0);
        out.tris.back() = Builder::bits(in.material);
        out.order[in.slot] = o;
    }
}

uint32_t max_split_picks(Light_tree const& tree, uint32_t start) {
    if (tree.num_nodes == 0) {
        return 0;
    }
    struct Walk {
        Light_tree const& t;
        uint32_t          count(uint32_t node, uint32_t depth) const {
            float const* n = &t.nodes[Light_node_floats * size_t(node)];
            uint32_t     first, lights;
            std::memcpy(&first, &n[9], 4);
            std::memcpy(&lights, &n[10], 4);
            if (lights != 0) {
                return depth < Max_split_depth ? lights : 1u;
            }
            if (depth >= Max_split_depth) {
                return 1u;
            }
            if (depth == Max_split_depth - 1) {
                return 2u;
            }
            return count(first, depth + 1) + count(first + 1, depth + 1);
        }
    };
    return Walk{tree}.count(0, start);
}

}  // namespace spb::render
