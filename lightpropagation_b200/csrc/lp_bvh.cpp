// lp_bvh.cpp -- binned-SAH BVH build on the host (see lp_bvh.hpp for the layout).
//
// The primitives (box, centroid, original index) are stored contiguously and partitioned
// in place, so every pass over a node reads memory in order.  The top levels of the tree
// are built by a parallel recursion (the two children of a node cover disjoint ranges of
// the primitive array, so one is built on a new thread) and the largest nodes bin their
// primitives on several threads.  Every split is decided as in a serial build and the
// nodes are renumbered breadth-first at the end, so the tree is the same for any thread
// count.
#include "lp_bvh.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <exception>
#include <thread>

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

struct Prim {
    Box box;
    float c[3];  // centroid of the box
    int32_t id;  // original triangle index
};

struct BNode {
    Box box;
    int32_t child[2] = {-1, -1};
    int64_t first = 0, count = 0;
    bool leaf = false;
};

constexpr int kBins = 32;

inline int bin_of(float x, float lo, double sc)
{
    const int b = (int)((x - lo) * sc);
    return std::min(std::max(b, 0), kBins - 1);
}

// Runs fn(k, lo, hi) over nt contiguous chunks of [0, n), chunk 0 on the calling thread.
// A chunk whose thread cannot be started runs on the calling thread instead (the build is
// called through the C ABI, where no exception may escape).
template <class Fn>
void for_chunks(int nt, int64_t n, Fn fn)
{
    std::vector<std::thread> pool;
    for (int k = 1; k < nt; ++k) {
        try {
            pool.emplace_back([&, k]() { fn(k, n * k / nt, n * (k + 1) / nt); });
        } catch (const std::exception &) {
            fn(k, n * k / nt, n * (k + 1) / nt);
        }
    }
    fn(0, 0, n / nt);
    for (std::thread &th : pool) th.join();
}

constexpr int64_t kParallelNode = 65536;  // nodes at least this large bin on several threads

// Computes the node's box and either marks it a leaf (returns false) or partitions its
// primitives at the best SAH bin boundary and returns true with `mid` the first index of
// the right half.  Min/max and integer counts merge exactly, so the chunked binning of
// large nodes gives the same bins as one pass.
bool split_node(Prim *pr, BNode &nd, int leaf_target, int64_t &mid, int n_threads)
{
    Box cb;  // centroid bounds
    nd.box = Box();
    Prim *const p0 = pr + nd.first, *const p1 = pr + nd.first + nd.count;
    const int nt = nd.count >= kParallelNode ? n_threads : 1;
    if (nt > 1) {
        std::vector<Box> part_box((size_t)nt), part_cb((size_t)nt);
        for_chunks(nt, nd.count, [&](int k, int64_t lo, int64_t hi) {
            Box b, c;  // local, so that the threads share no cache line while they scan
            for (const Prim *p = p0 + lo; p < p0 + hi; ++p) {
                b.grow(p->box);
                c.grow(p->c);
            }
            part_box[k] = b;
            part_cb[k] = c;
        });
        for (int k = 0; k < nt; ++k) {
            nd.box.grow(part_box[k]);
            cb.grow(part_cb[k]);
        }
    } else {
        for (const Prim *p = p0; p < p1; ++p) {
            nd.box.grow(p->box);
            cb.grow(p->c);
        }
    }
    bool make_leaf = nd.count <= leaf_target;
    int best_axis = -1, best_bin = -1;
    double best_cost = DBL_MAX;
    if (!make_leaf) {
        bool live[3];
        double sc[3];
        for (int a = 0; a < 3; ++a) {
            live[a] = cb.hi[a] > cb.lo[a];
            sc[a] = live[a] ? kBins / ((double)cb.hi[a] - cb.lo[a]) : 0.0;
        }
        struct Bins {
            Box bb[3][kBins];
            int64_t bc[3][kBins] = {};
        };
        auto bin_range = [&](Bins &B, const Prim *q0, const Prim *q1) {
            for (const Prim *p = q0; p < q1; ++p)
                for (int a = 0; a < 3; ++a) {
                    if (!live[a]) continue;
                    const int b = bin_of(p->c[a], cb.lo[a], sc[a]);
                    B.bb[a][b].grow(p->box);
                    B.bc[a][b]++;
                }
        };
        Bins all;
        if (nt > 1) {
            std::vector<Bins> part((size_t)nt);
            for_chunks(nt, nd.count, [&](int k, int64_t lo, int64_t hi) { bin_range(part[k], p0 + lo, p0 + hi); });
            for (int k = 0; k < nt; ++k)
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < kBins; ++b) {
                        all.bb[a][b].grow(part[k].bb[a][b]);
                        all.bc[a][b] += part[k].bc[a][b];
                    }
        } else {
            bin_range(all, p0, p1);
        }
        const auto &bb = all.bb;
        const auto &bc = all.bc;
        for (int a = 0; a < 3; ++a) {
            if (!live[a]) continue;
            double ra[kBins];
            int64_t rn[kBins];
            Box acc;
            int64_t cnt = 0;
            for (int b = kBins - 1; b > 0; --b) {
                acc.grow(bb[a][b]);
                cnt += bc[a][b];
                ra[b] = acc.area();
                rn[b] = cnt;
            }
            acc = Box();
            cnt = 0;
            for (int b = 0; b < kBins - 1; ++b) {
                acc.grow(bb[a][b]);
                cnt += bc[a][b];
                if (cnt == 0 || rn[b + 1] == 0) continue;
                const double c = acc.area() * (double)cnt + ra[b + 1] * (double)rn[b + 1];
                if (c < best_cost) {
                    best_cost = c;
                    best_axis = a;
                    best_bin = b;
                }
            }
        }
        const double leaf_cost = nd.box.area() * (double)nd.count;
        const double split_cost = nd.box.area() * 1.0 + best_cost;
        if (best_axis < 0 || (split_cost >= leaf_cost && nd.count <= kLeafMax)) make_leaf = nd.count <= kLeafMax;
    }
    if (make_leaf) {
        nd.leaf = true;
        return false;
    }
    if (best_axis >= 0) {
        const int a = best_axis;
        const float lo = cb.lo[a];
        const double sc = kBins / ((double)cb.hi[a] - lo);
        Prim *it = std::partition(p0, p1, [&](const Prim &p) { return bin_of(p.c[a], lo, sc) <= best_bin; });
        mid = nd.first + (it - p0);
    } else {
        mid = nd.first + nd.count / 2;  // coincident centroids: split by position in the list
    }
    if (mid == nd.first || mid == nd.first + nd.count) mid = nd.first + nd.count / 2;
    return true;
}

// Builds the subtree rooted at nodes[root] (first/count set), appending its nodes.
void build_from(Prim *pr, std::vector<BNode> &nodes, int32_t root, int leaf_target, int n_threads)
{
    std::vector<int32_t> work{root};
    while (!work.empty()) {
        const int32_t ni = work.back();
        work.pop_back();
        BNode nd = nodes[ni];
        int64_t mid = 0;
        if (!split_node(pr, nd, leaf_target, mid, n_threads)) {
            nodes[ni] = nd;
            continue;
        }
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
}

constexpr int64_t kParallelGrain = 4096;   // smaller subtrees are built where they are

// Builds the subtree over primitives [first, first + count) into `nodes` and returns its
// root's index.  While par_depth > 0 and the node is large, its right child is built on a
// new thread into a vector of its own, appended afterwards with shifted indices; the
// left child is built on this thread.  Every split is the one the serial build makes
// (split_node on the same primitive range), so the tree is the same.
int32_t build_par(Prim *pr, std::vector<BNode> &nodes, int64_t first, int64_t count, int leaf_target,
                  int par_depth, int bin_threads)
{
    const int32_t root = (int32_t)nodes.size();
    nodes.push_back(BNode());
    nodes[root].first = first;
    nodes[root].count = count;
    if (par_depth <= 0 || count < kParallelGrain) {
        build_from(pr, nodes, root, leaf_target, bin_threads);
        return root;
    }
    BNode nd = nodes[root];
    int64_t mid = 0;
    if (!split_node(pr, nd, leaf_target, mid, bin_threads)) {
        nodes[root] = nd;
        return root;
    }
    const int sub_bins = std::max(1, bin_threads / 2);
    std::vector<BNode> right;
    std::thread th;
    bool threaded = false;
    try {
        th = std::thread([&]() {
            build_par(pr, right, mid, first + count - mid, leaf_target, par_depth - 1, sub_bins);
        });
        threaded = true;
    } catch (const std::exception &) {
        // no thread to be had: the right child is built here after the left
    }
    nd.child[0] = build_par(pr, nodes, first, mid - first, leaf_target, par_depth - 1, sub_bins);
    if (threaded)
        th.join();
    else
        build_par(pr, right, mid, first + count - mid, leaf_target, par_depth - 1, sub_bins);
    const int32_t base = (int32_t)nodes.size();
    for (BNode b : right) {
        for (int c = 0; c < 2; ++c)
            if (b.child[c] >= 0) b.child[c] += base;
        nodes.push_back(b);
    }
    nd.child[1] = base;   // the right subtree's root is its vector's first node
    nodes[root] = nd;
    return root;
}

}  // namespace

void build_bvh(const float *tri, int64_t n, Bvh &out, int leaf_target, int threads)
{
    out = Bvh();
    std::vector<Prim> pr((size_t)n);
    Box scene;
    double max_abs = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const float *t = tri + 9 * i;
        Prim &p = pr[(size_t)i];
        for (int v = 0; v < 3; ++v) {
            p.box.grow(t + 3 * v);
            for (int a = 0; a < 3; ++a) max_abs = std::max(max_abs, (double)std::fabs(t[3 * v + a]));
        }
        for (int a = 0; a < 3; ++a) p.c[a] = 0.5f * (p.box.lo[a] + p.box.hi[a]);
        p.id = (int32_t)i;
        scene.grow(p.box);
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

    std::vector<BNode> nodes;
    nodes.reserve((size_t)(2 * n / std::max(1, leaf_target) + 4));
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int n_threads = threads > 0 ? std::min(threads, 64) : (int)std::min(hw, 16u);
    if (n < 32768 || n_threads == 1) {
        build_par(pr.data(), nodes, 0, n, leaf_target, 0, 1);
    } else {
        // enough levels of threads for about four subtrees per hardware thread
        int par_depth = 0;
        while ((1 << par_depth) < 4 * n_threads) ++par_depth;
        build_par(pr.data(), nodes, 0, n, leaf_target, par_depth, n_threads);
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
        const int32_t oi = pr[(size_t)j].id;
        const float *t = tri + 9 * (int64_t)oi;
        // E = K - M, F = L - M, exactly as FindTriangleInPath computes them
        float Ex = t[0] - t[6], Ey = t[1] - t[7], Ez = t[2] - t[8];
        float Fx = t[3] - t[6], Fy = t[4] - t[7], Fz = t[5] - t[8];
        float ob;
        std::memcpy(&ob, &oi, 4);
        // plane-distance factors: |(G x E) . F| * inv_n is the distance from a point to the
        // triangle's plane (G = point - M), and kappa * |G|_1 bounds the rounding of that
        // product in float (about 9 ulp of |G| |E| |F| / |E x F|, taken 10x larger here);
        // a degenerate triangle gets 0, 0, so its plane distance reads 0
        const double ex = Ex, ey = Ey, ez = Ez, fx = Fx, fy = Fy, fz = Fz;
        const double nx = ey * fz - ez * fy, ny = ez * fx - ex * fz, nz = ex * fy - ey * fx;
        const double nl = std::sqrt(nx * nx + ny * ny + nz * nz);
        const double el = std::sqrt(ex * ex + ey * ey + ez * ez), fl = std::sqrt(fx * fx + fy * fy + fz * fz);
        float inv_n = 0.0f, kappa = 0.0f;
        if (nl > 1e-30 * (el * fl + 1e-300) && std::isfinite(nl)) {
            inv_n = (float)((1.0 / nl) * (1.0 - 1e-6));
            kappa = (float)std::min(1e-5 * el * fl / nl, 1e30);
        }
        out.tri_a[j] = {t[6], t[7], t[8], Ex};
        out.tri_b[j] = {Ey, Ez, Fx, Fy};
        out.tri_c[j] = {Fz, ob, inv_n, kappa};
    }
}

}  // namespace lp
