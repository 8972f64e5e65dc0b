// lp_bvh.hpp -- SoA bounding-volume hierarchy over the triangle mesh.
//
// Replaces the brute-force O(T) scan of FindTriangleInPath
// (src/Simulation/MCLightPropagation.cl:1037-1093).  The device traversal returns
// exactly the triangle that scan returns: the same intersection arithmetic per
// triangle, the same strict/inclusive comparisons, and ties in distance broken
// towards the lower original index (the scan keeps the first of equal distances).
//
// Layout (binary tree, breadth-first node order so the top levels are a prefix
// that can be staged in shared memory):
//   node_a[i] = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)   child boxes of node i
//   node_b[i] = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   node_c[i] = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//   node_d[i] = (c0 ref, c1 ref, 0, 0): ref >= 0 internal node index,
//               ref < 0 leaf with ~ref = (first << 3) | (count - 1)
//   tri_a[j]  = (M.x, M.y, M.z, E.x)    triangle j in leaf order, E = K - M
//   tri_b[j]  = (E.y, E.z, F.x, F.y)    F = L - M
//   tri_c[j]  = (F.z, original index as int bits, inv_n, kappa): 1 / |E x F| and the
//               rounding factor of the plane distance |(G x E) . F| * inv_n (see build_bvh)
// Boxes are widened by a small absolute margin so that rounding in the ray/box
// test never culls a triangle the exact test accepts.
#pragma once
#include <cstdint>
#include <vector>

namespace lp {

struct F4 { float x, y, z, w; };
struct I4 { int32_t x, y, z, w; };

struct Bvh {
    std::vector<F4> node_a, node_b, node_c;
    std::vector<I4> node_d;
    std::vector<F4> tri_a, tri_b, tri_c;
    int32_t depth = 0;
    float margin = 0.0f;
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
};

constexpr int kLeafMax = 8;

// Builds the tree over n_tri triangles given as 9 floats (K, L, M) each.  threads: the
// worker threads of a large build (0: the hardware's, at most 16); the tree is the same
// for every thread count.
void build_bvh(const float *tri, int64_t n_tri, Bvh &out, int leaf_target = 4, int threads = 0);

}  // namespace lp
