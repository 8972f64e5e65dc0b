// Test harness: builds the BVH of lp_bvh.cpp over triangles read from a file and writes
// the tree out, so that tests/test_bvh_build.py can check it on a machine without a GPU.
//   bvh_dump <triangles.f32> <out.bin> [threads]
// Input: n x 9 float32 (K, L, M).  Output: int32 n_nodes, int32 n_tri, int32 depth,
// float32 margin, then node_a, node_b, node_c, node_d, tri_a, tri_b, tri_c (16 bytes each).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "lp_bvh.hpp"

int main(int argc, char **argv)
{
    if (argc != 3 && argc != 4) return 2;
    const int threads = argc == 4 ? std::atoi(argv[3]) : 0;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 3;
    std::vector<float> tri;
    float buf[4096];
    size_t k;
    while ((k = std::fread(buf, sizeof(float), 4096, f)) > 0) tri.insert(tri.end(), buf, buf + k);
    std::fclose(f);
    lp::Bvh b;
    lp::build_bvh(tri.data(), (int64_t)(tri.size() / 9), b, 4, threads);
    FILE *o = std::fopen(argv[2], "wb");
    if (!o) return 4;
    const int32_t hdr[3] = {(int32_t)b.node_a.size(), (int32_t)b.tri_a.size(), b.depth};
    std::fwrite(hdr, sizeof hdr, 1, o);
    std::fwrite(&b.margin, sizeof(float), 1, o);
    for (const auto *v : {&b.node_a, &b.node_b, &b.node_c}) std::fwrite(v->data(), 16, v->size(), o);
    std::fwrite(b.node_d.data(), 16, b.node_d.size(), o);
    for (const auto *v : {&b.tri_a, &b.tri_b, &b.tri_c}) std::fwrite(v->data(), 16, v->size(), o);
    std::fclose(o);
    return 0;
}
