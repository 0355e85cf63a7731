// Mesh trees of the FP32 forms (wavefront, adjoint, batch).
//
// The plain f64 form walks the reference's tree (src/bvh.rs:51-242: splits
// on the axis of largest centroid extent only, 8 bins, every leaf of at most
// 4 triangles), because its results must match the reference's bit for bit.
// The FP32 forms match the reference in distribution only, so they may walk
// any tree over the same triangles; the closest hit does not depend on the
// tree.  This one is a binned surface-area-heuristic tree over all three
// axes with leaves chosen by cost:
//
// * 16 bins per axis over the node's centroid box, the three axes binned in
//   one pass over the node's triangles;
// * a split's cost is kNodeCost + (area(left) * n_left + area(right) *
//   n_right) / area(node), a leaf's is its triangle count; a node of at most
//   kMaxLeaf triangles becomes a leaf when that is not dearer.  A child-pair
//   node visit is weighed as one triangle test: on the B200 the 1080p
//   mesh+env frame ran 3.23 / 3.23 / 3.25 / 3.25 / 3.23 / 3.18 / 3.10 G
//   paths/s at node costs 0.25 / 0.5 / 0.75 / 1 / 1.5 / 2 / 3 (at 0.5 and
//   below nearly every leaf holds one triangle: twice the nodes of 1);
// * kMaxLeaf = 6: the traversal's leaf code holds a count of 1 to 6 (7 marks
//   an instance, 0 the exit markers);
// * the children's boxes and centroid boxes are the merged boxes of their
//   bins, so each node's triangles are read twice (binning, partition);
// * the triangle boxes are the reference's (Aabb::from_points pads by 1e-9,
//   geometry.rs:70-80), so the FP32 node boxes carry the same margins.
//
// On the 1,310,720-triangle benchmark mesh, cast on the CPU (camera rays,
// cosine bounce rays from their hits, sun shadow rays), this tree visits
// about as many nodes as the reference's tree (+1-4%), 16-20% fewer leaves,
// and tests 53-55% fewer triangles per bounce and shadow ray.
//
// Subtrees above kParallelTris triangles build on their own threads; every
// subtree is emitted in preorder (a node, its left subtree, its right
// subtree) and the pieces are joined with their indices shifted, so the
// result does not depend on the thread count.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <future>
#include <limits>
#include <stdexcept>
#include <vector>

#include "host_scene.hpp"

namespace tpt {
namespace {

constexpr int kBins = 16;
constexpr int kMaxLeaf = 6;
constexpr double kNodeCost = 1.0;
constexpr size_t kParallelTris = 1 << 16;
constexpr int kParallelDepth = 6;  // at most 2^6 subtrees on their own threads

struct TBox {
    double lo[3], hi[3];
    static TBox none() {
        const double inf = std::numeric_limits<double>::infinity();
        return TBox{{inf, inf, inf}, {-inf, -inf, -inf}};
    }
    void merge(const TBox& b) {
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], b.lo[k]);
            hi[k] = std::max(hi[k], b.hi[k]);
        }
    }
    void grow(const double* p) {
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], p[k]);
            hi[k] = std::max(hi[k], p[k]);
        }
    }
    double half_area() const {
        const double x = std::max(0.0, hi[0] - lo[0]), y = std::max(0.0, hi[1] - lo[1]),
                     z = std::max(0.0, hi[2] - lo[2]);
        return x * y + y * z + z * x;
    }
};

struct Node {
    TBox box;
    int32_t left, right;  // -1 for a leaf
    uint32_t start, count;
    int32_t depth;
};

struct Bin {
    TBox box, cbox;
    int64_t n;
};

// A triangle's padded box, centroid and index, partitioned in place with
// the node ranges so that every pass over a range reads memory in order.
struct Prim {
    TBox box;
    double c[3];
    int64_t id;
};

struct Builder {
    std::vector<Prim>& prims;

    // Bin of centroid coordinate c in a centroid box that starts at lo
    // (scale = kBins / the box's extent).
    static int bin_of(double c, double lo, double scale) {
        int b = (int)((c - lo) * scale);
        return b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
    }

    // Appends the nodes of v to out, their child indices shifted; returns
    // the index of v's root.
    static int32_t append(std::vector<Node>& out, const std::vector<Node>& v) {
        const int32_t off = (int32_t)out.size();
        for (Node nd : v) {
            if (nd.left >= 0) { nd.left += off; nd.right += off; }
            out.push_back(nd);
        }
        return off;
    }

    // Appends the subtree over prims[s, e) to out in preorder.  box and cbox
    // are the merged triangle box and centroid box of the range.
    void build(size_t s, size_t e, const TBox& box, const TBox& cbox, int depth, std::vector<Node>& out) {
        const size_t n = e - s;
        const int32_t me = (int32_t)out.size();
        out.push_back(Node{box, -1, -1, (uint32_t)s, (uint32_t)n, depth});
        if (n <= 1) return;
        Bin bins[3][kBins];
        double scale[3];
        bool open[3];
        for (int ax = 0; ax < 3; ++ax) {
            const double ext = cbox.hi[ax] - cbox.lo[ax];
            open[ax] = ext > 0.0;
            scale[ax] = open[ax] ? kBins / ext : 0.0;
            for (Bin& b : bins[ax]) b = Bin{TBox::none(), TBox::none(), 0};
        }
        for (size_t k = s; k < e; ++k) {
            const Prim& p = prims[k];
            const double* c = p.c;
            for (int ax = 0; ax < 3; ++ax) {
                if (!open[ax]) continue;
                Bin& b = bins[ax][bin_of(c[ax], cbox.lo[ax], scale[ax])];
                b.box.merge(p.box);
                b.cbox.grow(c);
                ++b.n;
            }
        }
        double best = std::numeric_limits<double>::infinity();
        int bax = -1, bsplit = 0;
        for (int ax = 0; ax < 3; ++ax) {
            if (!open[ax]) continue;
            double right_cost[kBins];  // area * count of bins [i, kBins)
            TBox acc = TBox::none();
            int64_t cnt = 0;
            for (int i = kBins - 1; i >= 1; --i) {
                if (bins[ax][i].n) { acc.merge(bins[ax][i].box); cnt += bins[ax][i].n; }
                right_cost[i] = cnt ? acc.half_area() * (double)cnt : -1.0;
            }
            acc = TBox::none();
            cnt = 0;
            for (int i = 1; i < kBins; ++i) {
                if (bins[ax][i - 1].n) { acc.merge(bins[ax][i - 1].box); cnt += bins[ax][i - 1].n; }
                if (cnt == 0 || right_cost[i] < 0.0) continue;
                const double cost = acc.half_area() * (double)cnt + right_cost[i];
                if (cost < best) { best = cost; bax = ax; bsplit = i; }
            }
        }
        const double area = box.half_area();
        const double split_cost = bax < 0 ? std::numeric_limits<double>::infinity()
                                          : kNodeCost + (area > 0.0 ? best / area : (double)n);
        if (n <= (size_t)kMaxLeaf && (double)n <= split_cost) return;  // leaf

        size_t mid;
        TBox lb = TBox::none(), lcb = TBox::none(), rb = TBox::none(), rcb = TBox::none();
        if (bax >= 0) {
            const double lo = cbox.lo[bax], sc = scale[bax];
            const auto first_right = std::partition(prims.begin() + (ptrdiff_t)s, prims.begin() + (ptrdiff_t)e,
                                                    [&](const Prim& p) { return bin_of(p.c[bax], lo, sc) < bsplit; });
            mid = (size_t)(first_right - prims.begin());
            for (int i = 0; i < kBins; ++i) {
                const Bin& b = bins[bax][i];
                if (!b.n) continue;
                (i < bsplit ? lb : rb).merge(b.box);
                (i < bsplit ? lcb : rcb).merge(b.cbox);
            }
        } else {
            // every centroid of the range is the same point: halve the range
            mid = s + n / 2;
            for (size_t k = s; k < e; ++k) {
                (k < mid ? lb : rb).merge(prims[k].box);
                (k < mid ? lcb : rcb).grow(prims[k].c);
            }
        }
        if (mid == s || mid == e) throw std::logic_error("FP32 mesh tree: empty child");
        if (n >= kParallelTris && depth < kParallelDepth) {
            std::vector<Node> lv, rv;
            auto left = std::async(std::launch::async, [&] { build(s, mid, lb, lcb, depth + 1, lv); });
            build(mid, e, rb, rcb, depth + 1, rv);
            left.get();
            const int32_t l = append(out, lv);
            const int32_t r = append(out, rv);
            out[(size_t)me].left = l;
            out[(size_t)me].right = r;
        } else {
            const int32_t l = (int32_t)out.size();
            build(s, mid, lb, lcb, depth + 1, out);
            const int32_t r = (int32_t)out.size();
            build(mid, e, rb, rcb, depth + 1, out);
            out[(size_t)me].left = l;
            out[(size_t)me].right = r;
        }
        out[(size_t)me].start = 0;
        out[(size_t)me].count = 0;
    }
};

}  // namespace

HostBvh build_fp32_mesh_bvh(const double* positions, int64_t n_vertices, const int32_t* tri_idx, int64_t n_tris) {
    HostBvh out;
    const size_t nt = (size_t)n_tris;
    if (nt == 0) return out;
    if (n_tris >= (int64_t)1 << 31) throw std::runtime_error("mesh of 2^31 triangles or more");
    std::vector<Prim> prims(nt);
    TBox box = TBox::none(), cbox = TBox::none();
    for (size_t i = 0; i < nt; ++i) {
        TBox b = TBox::none();
        for (int k = 0; k < 3; ++k) {
            const int32_t vi = tri_idx[3 * i + k];
            if (vi < 0 || vi >= n_vertices) throw std::runtime_error("triangle vertex index out of range");
            b.grow(positions + 3 * (size_t)vi);
        }
        for (int k = 0; k < 3; ++k) { b.lo[k] = b.lo[k] - 1e-9; b.hi[k] = b.hi[k] + 1e-9; }
        Prim& p = prims[i];
        p.box = b;
        for (int k = 0; k < 3; ++k) p.c[k] = (b.lo[k] + b.hi[k]) * 0.5;
        p.id = (int64_t)i;
        box.merge(b);
        cbox.grow(p.c);
    }
    std::vector<Node> nodes;
    nodes.reserve(nt);
    Builder{prims}.build(0, nt, box, cbox, 1, nodes);
    out.indices.resize(nt);
    for (size_t i = 0; i < nt; ++i) out.indices[i] = prims[i].id;
    const size_t nn = nodes.size();
    out.bbox.resize(6 * nn);
    out.left_right.resize(2 * nn);
    out.start_count.resize(2 * nn);
    for (size_t i = 0; i < nn; ++i) {
        const Node& nd = nodes[i];
        for (int k = 0; k < 3; ++k) {
            out.bbox[6 * i + k] = nd.box.lo[k];
            out.bbox[6 * i + 3 + k] = nd.box.hi[k];
        }
        out.left_right[2 * i] = nd.left;
        out.left_right[2 * i + 1] = nd.right;
        out.start_count[2 * i] = nd.start;
        out.start_count[2 * i + 1] = nd.count;
        out.max_depth = std::max(out.max_depth, (int)nd.depth);
    }
    return out;
}

}  // namespace tpt
