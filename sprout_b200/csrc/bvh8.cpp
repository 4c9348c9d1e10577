// Host BVH construction for the GPU cast.
//
// 1. Binary tree by binned SAH (32 bins per axis over centroids, one primitive per leaf),
//    subtrees built in parallel.
// 2. Greedy collapse to 8-wide nodes: a wide node starts from one binary node's children and
//    repeatedly opens the child with the largest surface area until it has 8 children; a child
//    holding at most 3 triangles becomes a leaf slot, any other child a wide node of its own.
//    Wide nodes are emitted breadth first, so the top of the tree is one contiguous block.
// 3. Children are placed into slots so that, for a ray whose direction lies in octant o, slot
//    o holds the child that is nearest along that octant's diagonal; traversal visits slots in
//    the order o, o^1, o^2, ... (Ylitie, Karras and Laine, "Efficient Incoherent Ray Traversal
//    on GPUs Through Compressed Wide BVHs", HPG 2017, whose node encoding this follows).
// 4. Child boxes are padded by a small absolute margin and quantized outward to 8 bits, so
//    every stored box contains the triangle bounds widened by the hit margin (see cast.cu),
//    with room for the rounding of the traversal's slab arithmetic.
#include "bvh8.hpp"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <deque>
#include <limits>
#include <string>
#include <thread>

#include "common.hpp"

namespace spb {

namespace {

struct Box {
    float lo[3] = {std::numeric_limits<float>::max(), std::numeric_limits<float>::max(),
                   std::numeric_limits<float>::max()};
    float hi[3] = {-std::numeric_limits<float>::max(), -std::numeric_limits<float>::max(),
                   -std::numeric_limits<float>::max()};

    void grow(Box const& b) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], b.lo[a]);
            hi[a] = std::max(hi[a], b.hi[a]);
        }
    }

    void grow(float const* p) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], p[a]);
            hi[a] = std::max(hi[a], p[a]);
        }
    }

    bool empty() const {
        return lo[0] > hi[0];
    }

    float area() const {
        if (empty()) {
            return 0.f;
        }
        float const dx = hi[0] - lo[0];
        float const dy = hi[1] - lo[1];
        float const dz = hi[2] - lo[2];
        return 2.f * (dx * dy + dy * dz + dz * dx);
    }
};

struct Binary_node {
    Box      box;
    uint32_t left  = 0;  // first child (children are adjacent) or first primitive
    uint32_t count = 0;  // primitives in the subtree
    bool     leaf  = false;
};

constexpr uint32_t Num_bins             = 32;
constexpr uint32_t Parallel_threshold   = 1u << 15;
constexpr uint32_t Max_leaf_triangles   = 3;
// The collapse does not open a child holding at most Keep_leaf triangles: it stays one leaf
// slot of up to Keep_leaf triangles (0: every binary child with more than one triangle can be
// opened to fill the node).
#ifndef SPB_BVH_KEEP_LEAF
#define SPB_BVH_KEEP_LEAF 0
#endif
constexpr uint32_t Keep_leaf = SPB_BVH_KEEP_LEAF;
static_assert(Keep_leaf <= Max_leaf_triangles, "a kept leaf must fit one slot");

class Binary_builder {
  public:
    Binary_builder(std::vector<Box> const& boxes, std::vector<float> const& centroids,
                   uint32_t num_threads)
        : boxes_(boxes), centroids_(centroids), num_threads_(num_threads) {
        uint32_t const n = uint32_t(boxes.size());
        prims_.resize(n);
        for (uint32_t i = 0; i < n; ++i) {
            prims_[i] = i;
        }
        nodes_.resize(size_t(2) * n);
    }

    void build() {
        uint32_t const n = uint32_t(prims_.size());
        Box            box;
        Box            cbox;
        for (uint32_t i = 0; i < n; ++i) {
            box.grow(boxes_[i]);
            cbox.grow(&centroids_[3 * size_t(i)]);
        }
        next_node_ = 1;
        running_   = 1;
        build(0, 0, n, box, cbox, 0);
        nodes_.resize(next_node_.load());
    }

    std::vector<Binary_node>& nodes() {
        return nodes_;
    }

    std::vector<uint32_t> const& prims() const {
        return prims_;
    }

  private:
    struct Bin {
        Box      box;
        Box      cbox;
        uint32_t count = 0;
    };

    void build(uint32_t node_id, uint32_t begin, uint32_t end, Box const& box, Box const& cbox,
               uint32_t depth) {
        Binary_node& node = nodes_[node_id];
        node.box          = box;
        node.count        = end - begin;

        if (end - begin == 1) {
            node.leaf = true;
            node.left = begin;
            return;
        }

        uint32_t mid = begin;
        Box      lbox;
        Box      rbox;
        Box      lcbox;
        Box      rcbox;

        if (!split(begin, end, cbox, mid, lbox, rbox, lcbox, rcbox)) {
            // All centroids coincide: split the range in half.
            mid = begin + (end - begin) / 2;
            for (uint32_t i = begin; i < mid; ++i) {
                lbox.grow(boxes_[prims_[i]]);
                lcbox.grow(&centroids_[3 * size_t(prims_[i])]);
            }
            for (uint32_t i = mid; i < end; ++i) {
                rbox.grow(boxes_[prims_[i]]);
                rcbox.grow(&centroids_[3 * size_t(prims_[i])]);
            }
        }

        uint32_t const child = next_node_.fetch_add(2);
        node.leaf            = false;
        node.left            = child;

        bool const parallel = (end - begin) >= Parallel_threshold &&
                              running_.load() < num_threads_;
        if (parallel) {
            running_.fetch_add(1);
            std::thread worker([this, child, begin, mid, lbox, lcbox, depth]() {
                build(child, begin, mid, lbox, lcbox, depth + 1);
                running_.fetch_sub(1);
            });
            build(child + 1, mid, end, rbox, rcbox, depth + 1);
            worker.join();
        } else {
            build(child, begin, mid, lbox, lcbox, depth + 1);
            build(child + 1, mid, end, rbox, rcbox, depth + 1);
        }
    }

    // Binned SAH over the centroid bounds on all three axes.  Partitions prims_[begin, end)
    // and returns the child bounds; false if no axis has a centroid extent.
    bool split(uint32_t begin, uint32_t end, Box const& cbox, uint32_t& mid, Box& lbox,
               Box& rbox, Box& lcbox, Box& rcbox) {
        float best_cost = std::numeric_limits<float>::max();
        int   best_axis = -1;
        int   best_bin  = 0;

        Bin bins[3][Num_bins];

        float scale[3];
        for (int a = 0; a < 3; ++a) {
            float const extent = cbox.hi[a] - cbox.lo[a];
            scale[a]           = extent > 0.f ? float(Num_bins) / extent : 0.f;
        }

        for (uint32_t i = begin; i < end; ++i) {
            uint32_t const p = prims_[i];
            float const*   c = &centroids_[3 * size_t(p)];
            for (int a = 0; a < 3; ++a) {
                if (scale[a] == 0.f) {
                    continue;
                }
                uint32_t const b = bin_of(c[a], cbox.lo[a], scale[a]);
                bins[a][b].count++;
                bins[a][b].box.grow(boxes_[p]);
                bins[a][b].cbox.grow(c);
            }
        }

        for (int a = 0; a < 3; ++a) {
            if (scale[a] == 0.f) {
                continue;
            }
            float    right_area[Num_bins];
            uint32_t right_count[Num_bins];
            Box      acc;
            uint32_t cnt = 0;
            for (int b = int(Num_bins) - 1; b > 0; --b) {
                acc.grow(bins[a][b].box);
                cnt += bins[a][b].count;
                right_area[b]  = acc.area();
                right_count[b] = cnt;
            }
            acc = Box();
            cnt = 0;
            for (uint32_t b = 1; b < Num_bins; ++b) {
                acc.grow(bins[a][b - 1].box);
                cnt += bins[a][b - 1].count;
                if (cnt == 0 || right_count[b] == 0) {
                    continue;
                }
                float const cost = acc.area() * float(cnt) + right_area[b] * float(right_count[b]);
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = a;
                    best_bin  = int(b);
                }
            }
        }

        if (best_axis < 0) {
            return false;
        }

        int const   a  = best_axis;
        float const lo = cbox.lo[a];
        float const sc = scale[a];
        auto* const it = std::partition(prims_.data() + begin, prims_.data() + end,
                                        [&](uint32_t p) {
                                            return int(bin_of(centroids_[3 * size_t(p) + a], lo,
                                                              sc)) < best_bin;
                                        });
        mid = uint32_t(it - prims_.data());
        for (int b = 0; b < best_bin; ++b) {
            lbox.grow(bins[a][b].box);
            lcbox.grow(bins[a][b].cbox);
        }
        for (int b = best_bin; b < int(Num_bins); ++b) {
            rbox.grow(bins[a][b].box);
            rcbox.grow(bins[a][b].cbox);
        }
        return mid > begin && mid < end;
    }

    static uint32_t bin_of(float c, float lo, float scale) {
        float const    f = (c - lo) * scale;
        uint32_t const b = f <= 0.f ? 0u : uint32_t(f);
        return std::min(b, Num_bins - 1);
    }

    std::vector<Box> const&   boxes_;
    std::vector<float> const& centroids_;
    uint32_t                  num_threads_;

    std::vector<uint32_t>    prims_;
    std::vector<Binary_node> nodes_;
    std::atomic<uint32_t>    next_node_{0};
    std::atomic<uint32_t>    running_{0};
};

// Smallest e with 255 * 2^e >= extent, clamped to the normal float exponent range.
int32_t quant_exponent(double extent) {
    if (!(extent > 0.)) {
        return -126;
    }
    int32_t e = int32_t(std::ceil(std::log2(extent / 255.)));
    while (std::ldexp(255., e) < extent) {
        ++e;
    }
    while (e > -126 && std::ldexp(255., e - 1) >= extent) {
        --e;
    }
    return std::clamp(e, -126, 127);
}

float round_down(double x) {
    float f = float(x);
    if (double(f) > x) {
        f = std::nextafter(f, -std::numeric_limits<float>::infinity());
    }
    return f;
}

}  // namespace

double scene_box_pad(double extent, double magnitude) {
    return std::max(std::ldexp(std::max(extent, magnitude), -10), double(FLT_MIN));
}

float hit_margin_for(double extent, double magnitude) {
    float const m = float(std::ldexp(std::max(extent, magnitude), -17));
    return m > std::numeric_limits<float>::min() ? m : std::numeric_limits<float>::min();
}

// Binary SAH tree over the primitives' boxes, collapsed to 8-wide nodes; emit(p, record)
// fills the leaf record of primitive p.
template <typename Emit>
bool collapse_tree(std::vector<Box> const& boxes, std::vector<float> const& centroids,
                   uint32_t num_threads, Wide_bvh& out, std::string& error, Emit&& emit) {
    Binary_builder builder(boxes, centroids, num_threads);
    builder.build();
    auto&       bnodes = builder.nodes();
    auto const& prims  = builder.prims();

    Box const& root_box = bnodes[0].box;
    double     extent   = 0.;
    double     magnitude = 0.;
    for (int a = 0; a < 3; ++a) {
        extent    = std::max(extent, double(root_box.hi[a]) - double(root_box.lo[a]));
        magnitude = std::max({magnitude, std::fabs(double(root_box.lo[a])),
                              std::fabs(double(root_box.hi[a]))});
    }
    // A hit counts only if its point lies within the triangle's bounds widened by
    // hit_margin (2^-17 of the scene size); child boxes are widened by twice that, which
    // leaves hit_margin of room for the rounding of the traversal's slab arithmetic.
    out.hit_margin   = hit_margin_for(extent, magnitude);
    double const pad = 2.0 * double(out.hit_margin);
    double const scene_pad = scene_box_pad(extent, magnitude);
    for (int a = 0; a < 3; ++a) {
        out.scene_lo[a] = std::nextafter(float(double(root_box.lo[a]) - scene_pad), -INFINITY);
        out.scene_hi[a] = std::nextafter(float(double(root_box.hi[a]) + scene_pad), INFINITY);
    }

    double const root_area = std::max(double(root_box.area()), 1e-30);

    // Collapse.  Each queue entry is a wide node to fill from a binary node.
    struct Pending {
        uint32_t wide;
        uint32_t binary;
        uint32_t depth;
    };
    std::deque<Pending> queue;
    out.nodes.emplace_back();
    queue.push_back({0, 0, 1});

    auto gather = [&](uint32_t b, std::vector<uint32_t>& tris) {
        std::vector<uint32_t> stack{b};
        while (!stack.empty()) {
            uint32_t const n = stack.back();
            stack.pop_back();
            if (bnodes[n].leaf) {
                for (uint32_t i = 0; i < bnodes[n].count; ++i) {
                    tris.push_back(prims[bnodes[n].left + i]);
                }
            } else {
                stack.push_back(bnodes[n].left + 1);
                stack.push_back(bnodes[n].left);
            }
        }
    };

    while (!queue.empty()) {
        Pending const job = queue.front();
        queue.pop_front();
        out.max_depth = std::max(out.max_depth, job.depth);

        // Children of this wide node, as binary nodes.
        std::vector<uint32_t> kids;
        Binary_node const&    src = bnodes[job.binary];
        if (src.leaf || src.count <= Max_leaf_triangles) {
            kids.push_back(job.binary);
        } else {
            kids.push_back(src.left);
            kids.push_back(src.left + 1);
            while (kids.size() < 8) {
                int   best      = -1;
                float best_area = -1.f;
                for (size_t i = 0; i < kids.size(); ++i) {
                    Binary_node const& k = bnodes[kids[i]];
                    if (k.leaf || k.count <= Keep_leaf) {
                        continue;
                    }
                    float const a = k.box.area();
                    if (a > best_area) {
                        best_area = a;
                        best      = int(i);
                    }
                }
                if (best < 0) {
                    break;
                }
                uint32_t const opened = kids[size_t(best)];
                kids[size_t(best)]    = bnodes[opened].left;
                kids.push_back(bnodes[opened].left + 1);
            }
        }

        size_t const nk = kids.size();

        // Octant slot assignment: slot s takes the child nearest along diagonal dir(s).
        Box node_box;
        for (uint32_t k : kids) {
            node_box.grow(bnodes[k].box);
        }
        float pc[3];
        for (int a = 0; a < 3; ++a) {
            pc[a] = 0.5f * (node_box.lo[a] + node_box.hi[a]);
        }
        float cost[8][8];
        for (size_t c = 0; c < nk; ++c) {
            Box const& b = bnodes[kids[c]].box;
            float      d[3];
            for (int a = 0; a < 3; ++a) {
                d[a] = 0.5f * (b.lo[a] + b.hi[a]) - pc[a];
            }
            for (int s = 0; s < 8; ++s) {
                float const sx = (s & 1) ? -1.f : 1.f;
                float const sy = (s & 2) ? -1.f : 1.f;
                float const sz = (s & 4) ? -1.f : 1.f;
                cost[c][s]     = d[0] * sx + d[1] * sy + d[2] * sz;
            }
        }
        int  slot_of[8];
        int  child_in[8];
        bool used_child[8] = {};
        for (int s = 0; s < 8; ++s) {
            child_in[s] = -1;
        }
        for (size_t round = 0; round < nk; ++round) {
            float best = std::numeric_limits<float>::max();
            int   bc   = -1;
            int   bs   = -1;
            for (size_t c = 0; c < nk; ++c) {
                if (used_child[c]) {
                    continue;
                }
                for (int s = 0; s < 8; ++s) {
                    if (child_in[s] >= 0) {
                        continue;
                    }
                    if (cost[c][s] < best || bc < 0) {
                        best = cost[c][s];
                        bc   = int(c);
                        bs   = s;
                    }
                }
            }
            used_child[bc] = true;
            child_in[bs]   = bc;
            slot_of[bc]    = bs;
        }
        (void)slot_of;

        // Quantization frame: padded node box, origin rounded down to float.
        float    origin[3];
        int32_t  expo[3];
        double   scale[3];
        for (int a = 0; a < 3; ++a) {
            double const lo = double(node_box.lo[a]) - pad;
            double const hi = double(node_box.hi[a]) + pad;
            origin[a]       = round_down(lo);
            expo[a]         = quant_exponent(hi - double(origin[a]));
            scale[a]        = std::ldexp(1., expo[a]);
        }

        Wide_node wn;
        std::memset(&wn, 0, sizeof(wn));
        for (int a = 0; a < 3; ++a) {
            wn.origin[a]   = origin[a];
            wn.exponent[a] = uint8_t(expo[a] + 127);
        }
        wn.child_base = uint32_t(out.nodes.size());
        wn.tri_base   = uint32_t(out.triangles.size());

        double node_area = double(node_box.area());
        out.sah_cost += node_area / root_area;

        uint32_t tri_offset = 0;
        for (int s = 0; s < 8; ++s) {
            int const c = child_in[s];
            if (c < 0) {
                // Empty slot: inverted box, no meta bits.
                for (int a = 0; a < 3; ++a) {
                    wn.qlo[a][s] = 255;
                    wn.qhi[a][s] = 0;
                }
                continue;
            }
            Binary_node const& b = bnodes[kids[size_t(c)]];
            for (int a = 0; a < 3; ++a) {
                double const lo = (double(b.box.lo[a]) - pad - double(origin[a])) / scale[a];
                double const hi = (double(b.box.hi[a]) + pad - double(origin[a])) / scale[a];
                wn.qlo[a][s]    = uint8_t(std::clamp(std::floor(lo), 0., 255.));
                wn.qhi[a][s]    = uint8_t(std::clamp(std::ceil(hi), 0., 255.));
            }
            if (b.count <= Max_leaf_triangles) {
                std::vector<uint32_t> tris;
                gather(kids[size_t(c)], tris);
                uint32_t const cnt = uint32_t(tris.size());
                wn.meta[s] = uint8_t((((1u << cnt) - 1u) << 5) | tri_offset);
                for (uint32_t t : tris) {
                    Wide_triangle wt;
                    std::memset(&wt, 0, sizeof(wt));
                    emit(t, wt);
                    out.triangles.push_back(wt);
                }
                tri_offset += cnt;
                out.num_leaves++;
                out.sah_cost += double(b.box.area()) / root_area * double(cnt);
            } else {
                wn.imask |= uint8_t(1u << s);
                wn.meta[s] = uint8_t((1u << 5) | (24u + uint32_t(s)));
            }
        }

        // Internal children, contiguous from child_base in slot order.
        for (int s = 0; s < 8; ++s) {
            if (wn.imask & (1u << s)) {
                uint32_t const w = uint32_t(out.nodes.size());
                out.nodes.emplace_back();
                queue.push_back({w, kids[size_t(child_in[s])], job.depth + 1});
            }
        }
        out.nodes[job.wide] = wn;
    }

    if (out.max_depth > Max_wide_depth) {
        error = "tree deeper than the traversal stack (" + std::to_string(out.max_depth) + ")";
        return false;
    }
    return true;
}

bool build_wide_bvh(uint32_t num_vertices, uint32_t num_triangles, float const* positions,
                    uint32_t const* indices, uint32_t num_threads, Wide_bvh& out,
                    std::string& error, uint32_t const* tri_class) {
    out = Wide_bvh();

    if (num_triangles == 0) {
        error = "mesh has no triangles";
        return false;
    }
    for (uint64_t i = 0; i < uint64_t(num_triangles) * 3; ++i) {
        if (indices[i] >= num_vertices) {
            error = "triangle index out of range";
            return false;
        }
    }

    std::vector<Box>   boxes(num_triangles);
    std::vector<float> centroids(size_t(num_triangles) * 3);
    parallel_ranges(num_triangles, num_threads, [&](uint32_t, uint64_t begin, uint64_t end) {
        for (uint64_t t = begin; t < end; ++t) {
            Box b;
            for (int k = 0; k < 3; ++k) {
                b.grow(positions + 3 * size_t(indices[3 * t + k]));
            }
            boxes[t] = b;
            for (int a = 0; a < 3; ++a) {
                centroids[3 * t + a] = 0.5f * (b.lo[a] + b.hi[a]);
            }
        }
    });

    for (uint32_t t = 0; t < num_triangles; ++t) {
        for (int a = 0; a < 3; ++a) {
            if (!std::isfinite(boxes[t].lo[a]) || !std::isfinite(boxes[t].hi[a])) {
                error = "mesh has non-finite vertex positions";
                return false;
            }
        }
    }

    return collapse_tree(boxes, centroids, num_threads, out, error,
                         [&](uint32_t t, Wide_triangle& wt) {
                             float const* pa = positions + 3 * size_t(indices[3 * size_t(t) + 0]);
                             float const* pb = positions + 3 * size_t(indices[3 * size_t(t) + 1]);
                             float const* pc = positions + 3 * size_t(indices[3 * size_t(t) + 2]);
                             for (int a = 0; a < 3; ++a) {
                                 wt.a[a]  = pa[a];
                                 wt.e1[a] = pb[a] - pa[a];
                                 wt.e2[a] = pc[a] - pa[a];
                             }
                             wt.id        = t;
                             wt.tri_class = tri_class ? tri_class[t] : 0u;
                         });
}

bool build_wide_instances(uint32_t num_instances, float const* boxes_lo_hi, uint32_t instance_class,
                          uint32_t num_threads, Wide_bvh& out, std::string& error) {
    out = Wide_bvh();
    if (num_instances == 0) {
        error = "no instances";
        return false;
    }
    std::vector<Box>   boxes(num_instances);
    std::vector<float> centroids(size_t(num_instances) * 3);
    for (uint32_t i = 0; i < num_instances; ++i) {
        boxes[i].grow(boxes_lo_hi + 6 * size_t(i));
        boxes[i].grow(boxes_lo_hi + 6 * size_t(i) + 3);
        for (int a = 0; a < 3; ++a) {
            if (!std::isfinite(boxes[i].lo[a]) || !std::isfinite(boxes[i].hi[a])) {
                error = "instance with non-finite bounds";
                return false;
            }
            centroids[3 * size_t(i) + a] = 0.5f * (boxes[i].lo[a] + boxes[i].hi[a]);
        }
    }
    return collapse_tree(boxes, centroids, num_threads, out, error,
                         [&](uint32_t i, Wide_triangle& wt) {
                             wt.id        = i;
                             wt.tri_class = instance_class;
                         });
}


}  // namespace spb
