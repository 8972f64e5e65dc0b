// lp_bvh.cpp -- binned-SAH BVH build on the host (see lp_bvh.hpp for the layout).
#include "lp_bvh.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

namespace lp {
namespace {

struct Box {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void grow(const Box &b)
    {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], b.lo[a]);
            hi[a] = std::max(hi[a], b.hi[a]);
        }
    }
    void grow(const float *p)
    {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], p[a]);
            hi[a] = std::max(hi[a], p[a]);
        }
    }
    bool empty() const { return lo[0] > hi[0]; }
    double area() const
    {
        if (empty()) return 0.0;
        double dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        return 2.0 * (dx * dy + dy * dz + dz * dx);
    }
};

struct BNode {
    Box box;
    int32_t child[2] = {-1, -1};
    int64_t first = 0, count = 0;
    bool leaf = false;
};

constexpr int kBins = 32;

}  // namespace

void build_bvh(const float *tri, int64_t n, Bvh &out, int leaf_target)
{
    out = Bvh();
    std::vector<Box> tb((size_t)n);
    std::vector<float> cen((size_t)n * 3);
    Box scene;
    double max_abs = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const float *t = tri + 9 * i;
        for (int v = 0; v < 3; ++v) {
            tb[i].grow(t + 3 * v);
            for (int a = 0; a < 3; ++a) max_abs = std::max(max_abs, (double)std::fabs(t[3 * v + a]));
        }
        for (int a = 0; a < 3; ++a) cen[3 * i + a] = 0.5f * (tb[i].lo[a] + tb[i].hi[a]);
        scene.grow(tb[i]);
    }
    double ext = 0.0;
    if (n > 0)
        for (int a = 0; a < 3; ++a) ext = std::max(ext, (double)scene.hi[a] - scene.lo[a]);
    const float margin = (float)(1e-5 * std::max(ext, max_abs) + 1e-30);
    out.margin = margin;
    for (int a = 0; a < 3; ++a) {
        out.lo[a] = n ? scene.lo[a] : 0.0f;
        out.hi[a] = n ? scene.hi[a] : 0.0f;
    }

    std::vector<int64_t> idx((size_t)n);
    for (int64_t i = 0; i < n; ++i) idx[i] = i;
    std::vector<BNode> nodes;
    nodes.reserve((size_t)(2 * n / std::max(1, leaf_target) + 4));
    nodes.push_back(BNode());
    nodes[0].first = 0;
    nodes[0].count = n;
    std::vector<int32_t> work{0};
    while (!work.empty()) {
        int32_t ni = work.back();
        work.pop_back();
        BNode nd = nodes[ni];
        Box cb;  // centroid bounds
        nd.box = Box();
        for (int64_t k = nd.first; k < nd.first + nd.count; ++k) {
            nd.box.grow(tb[idx[k]]);
            cb.grow(&cen[3 * idx[k]]);
        }
        bool make_leaf = nd.count <= leaf_target;
        int best_axis = -1, best_bin = -1;
        double best_cost = DBL_MAX;
        if (!make_leaf) {
            for (int a = 0; a < 3; ++a) {
                float lo = cb.lo[a], hi = cb.hi[a];
                if (!(hi > lo)) continue;
                Box bb[kBins];
                int64_t bc[kBins] = {0};
                const double sc = kBins / ((double)hi - lo);
                for (int64_t k = nd.first; k < nd.first + nd.count; ++k) {
                    int b = (int)((cen[3 * idx[k] + a] - lo) * sc);
                    b = std::min(std::max(b, 0), kBins - 1);
                    bb[b].grow(tb[idx[k]]);
                    bc[b]++;
                }
                double ra[kBins];
                int64_t rn[kBins];
                Box acc;
                int64_t cnt = 0;
                for (int b = kBins - 1; b > 0; --b) {
                    acc.grow(bb[b]);
                    cnt += bc[b];
                    ra[b] = acc.area();
                    rn[b] = cnt;
                }
                acc = Box();
                cnt = 0;
                for (int b = 0; b < kBins - 1; ++b) {
                    acc.grow(bb[b]);
                    cnt += bc[b];
                    if (cnt == 0 || rn[b + 1] == 0) continue;
                    double c = acc.area() * (double)cnt + ra[b + 1] * (double)rn[b + 1];
                    if (c < best_cost) {
                        best_cost = c;
                        best_axis = a;
                        best_bin = b;
                    }
                }
            }
            double leaf_cost = nd.box.area() * (double)nd.count;
            double split_cost = nd.box.area() * 1.0 + best_cost;
            if (best_axis < 0 || (split_cost >= leaf_cost && nd.count <= kLeafMax)) make_leaf = nd.count <= kLeafMax;
        }
        if (make_leaf) {
            nd.leaf = true;
            nodes[ni] = nd;
            continue;
        }
        int64_t mid;
        if (best_axis >= 0) {
            float lo = cb.lo[best_axis], hi = cb.hi[best_axis];
            const double sc = kBins / ((double)hi - lo);
            auto it = std::partition(idx.begin() + nd.first, idx.begin() + nd.first + nd.count,
                                     [&](int64_t t) {
                                         int b = (int)((cen[3 * t + best_axis] - lo) * sc);
                                         b = std::min(std::max(b, 0), kBins - 1);
                                         return b <= best_bin;
                                     });
            mid = it - idx.begin();
        } else {
            mid = nd.first + nd.count / 2;  // coincident centroids: split by position in the list
        }
        if (mid == nd.first || mid == nd.first + nd.count) mid = nd.first + nd.count / 2;
        BNode l, r;
        l.first = nd.first;
        l.count = mid - nd.first;
        r.first = mid;
        r.count = nd.first + nd.count - mid;
        nd.child[0] = (int32_t)nodes.size();
        nd.child[1] = (int32_t)nodes.size() + 1;
        nodes[ni] = nd;
        nodes.push_back(l);
        nodes.push_back(r);
        work.push_back(nd.child[1]);
        work.push_back(nd.child[0]);
    }

    // A root that is a leaf gets a synthetic internal parent whose two children are
    // that same leaf (testing a triangle twice cannot change the (t, index) minimum).
    int32_t root = 0;
    if (nodes[0].leaf) {
        BNode wrap;
        wrap.child[0] = 0;
        wrap.child[1] = 0;
        wrap.box = nodes[0].box;
        nodes.push_back(wrap);
        root = (int32_t)nodes.size() - 1;
    }
    // breadth-first numbering of internal nodes
    std::vector<int32_t> order{root};
    std::vector<int32_t> level{0};
    std::vector<int32_t> newid(nodes.size(), -1);
    for (size_t q = 0; q < order.size(); ++q) {
        newid[order[q]] = (int32_t)q;
        for (int c = 0; c < 2; ++c) {
            int32_t ch = nodes[order[q]].child[c];
            if (ch >= 0 && !nodes[ch].leaf) {
                order.push_back(ch);
                level.push_back(level[q] + 1);
            }
        }
    }
    out.depth = 0;
    for (int32_t l : level) out.depth = std::max(out.depth, l + 1);
    const size_t nn = order.size();
    out.node_a.resize(nn);
    out.node_b.resize(nn);
    out.node_c.resize(nn);
    out.node_d.resize(nn);
    auto child_box = [&](int32_t ch, float lo[3], float hi[3]) {
        const BNode &c = nodes[ch];
        for (int a = 0; a < 3; ++a) {
            lo[a] = c.box.lo[a] - margin;
            hi[a] = c.box.hi[a] + margin;
        }
    };
    auto child_ref = [&](int32_t ch) -> int32_t {
        const BNode &c = nodes[ch];
        if (!c.leaf) return newid[ch];
        return ~(int32_t)((c.first << 3) | (c.count - 1));
    };
    for (size_t q = 0; q < nn; ++q) {
        const BNode &nd = nodes[order[q]];
        float l0[3], h0[3], l1[3], h1[3];
        child_box(nd.child[0], l0, h0);
        child_box(nd.child[1], l1, h1);
        out.node_a[q] = {l0[0], h0[0], l0[1], h0[1]};
        out.node_b[q] = {l1[0], h1[0], l1[1], h1[1]};
        out.node_c[q] = {l0[2], h0[2], l1[2], h1[2]};
        out.node_d[q] = {child_ref(nd.child[0]), child_ref(nd.child[1]), 0, 0};
    }
    out.tri_a.resize((size_t)n);
    out.tri_b.resize((size_t)n);
    out.tri_c.resize((size_t)n);
    for (int64_t j = 0; j < n; ++j) {
        const int64_t o = idx[j];
        const float *t = tri + 9 * o;
        // E = K - M, F = L - M, exactly as FindTriangleInPath computes them
        float Ex = t[0] - t[6], Ey = t[1] - t[7], Ez = t[2] - t[8];
        float Fx = t[3] - t[6], Fy = t[4] - t[7], Fz = t[5] - t[8];
        int32_t oi = (int32_t)o;
        float ob;
        std::memcpy(&ob, &oi, 4);
        out.tri_a[j] = {t[6], t[7], t[8], Ex};
        out.tri_b[j] = {Ey, Ez, Fx, Fy};
        out.tri_c[j] = {Fz, ob, 0.0f, 0.0f};
    }
}

}  // namespace lp
