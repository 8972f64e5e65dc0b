/*
 * ref_entry.cpp -- C entry points around the reference kernel compiled for the CPU.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/build_ref.py compiles this file together with
 * the reference's own sources (src/Simulation/MCLightPropagation.cl, after the
 * vector-literal rewrite, and src/PSNR/PSNR.cpp) into oracle/_ref/libclref.so.
 * The resulting library is the pin for lp_oracle.c; it is never shipped.
 */
#include "clshim.hpp"
#include <thread>
#include <vector>

#define __kernel
#define __global
#define __local
#define __constant
#define __private
#define global

namespace clref {
thread_local long g_global_id = 0;
long g_global_size = 1;
#include LP_CL_SOURCE
} // namespace clref

#undef global
#undef __kernel
#undef __global
#undef __local
#undef __constant
#undef __private

#include LP_PSNR_HEADER

extern "C" {

/* PSNR::SetSeed + InitRand3 + GetRan3Array + GetInextInextp (PSNR.cpp:80-237). */
void clref_psnr_state(int seed, float *state56, int *inext3)
{
    PSNR *r = new PSNR;
    r->SetSeed(seed);
    r->InitRand3();
    std::vector<float> a;
    std::vector<int> ix;
    r->GetRan3Array(a);
    r->GetInextInextp(ix);
    for (int i = 0; i < 56; ++i) state56[i] = a[i];
    state56[0] = 0.0f; /* ma[0] is never initialised by PSNR and never read by the kernel */
    for (int i = 0; i < 3; ++i) inext3[i] = ix[i];
    delete r;
}

/* Runs work-items 0..n_items-1 of MCLightPropagation one after another with the
 * argument list of MCLightPropagation.cl:1262-1269.  Buffers are caller-owned;
 * mesh arrays and the r-z buffer must be padded so that the reference's
 * out-of-range indices (mediumIDs[-1] on a miss, r-z cells beyond the image)
 * stay inside the allocation. */
int clref_run(int numTriangles, float factor, const float *vStart, const int *vStartOcc,
              const float *pStart3, float chance, float w_threshold, int fetalTissueID,
              float *SurfFetalTransRxyG, float *RecordAxzAyz, const float *dimsXYZ,
              const float *e_P0XYZ, const float *gridDims, float *triangles, float *normals,
              const int *mediumIDs, const float *nMuasG, float *rand3Arr, int *inxtInxtpLocked,
              long n_items)
{
    clref::float3 pStart(pStart3[0], pStart3[1], pStart3[2]);
    clref::g_global_size = n_items;
    for (long i = 0; i < n_items; ++i) {
        clref::g_global_id = i;
        clref::MCLightPropagation(numTriangles, factor, vStart, vStartOcc, pStart, chance,
                                  w_threshold, fetalTissueID, SurfFetalTransRxyG, RecordAxzAyz,
                                  dimsXYZ, e_P0XYZ, gridDims, triangles, normals, mediumIDs,
                                  nMuasG, rand3Arr, inxtInxtpLocked);
    }
    return 0;
}

/* CPU baseline driver: n_items work-items over nthreads host threads.  Each thread
 * plays one OpenCL work-group of the reference: it starts from the same copy of the
 * ran3 table (every work-group of a launch does, MCLightPropagation.cl:1316-1317),
 * runs its work-items one after another and writes its exit records; each thread
 * has its own r-z buffer (rz_cells floats x3 each, caller-allocated nthreads times).
 * Returns 0. */
int clref_run_mt(int numTriangles, float factor, const float *vStart, const int *vStartOcc,
                 const float *pStart3, float chance, float w_threshold, int fetalTissueID,
                 float *SurfFetalTransRxyG, float *rz_buffers, long rz_stride_cells, long rz_offset_cells,
                 const float *dimsXYZ, const float *e_P0XYZ, const float *gridDims, float *triangles,
                 float *normals, const int *mediumIDs, const float *nMuasG, const float *rand3Arr0,
                 const int *inxt0, long n_items, int nthreads)
{
    clref::float3 pStart(pStart3[0], pStart3[1], pStart3[2]);
    clref::g_global_size = n_items;
    if (nthreads < 1) nthreads = 1;
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t) {
        th.emplace_back([=]() {
            float st[56];
            int ix[3];
            for (int i = 0; i < 56; ++i) st[i] = rand3Arr0[i];
            for (int i = 0; i < 3; ++i) ix[i] = inxt0[i];
            float *rz = rz_buffers + 3 * (rz_stride_cells * t + rz_offset_cells);
            const long lo = n_items * t / nthreads, hi = n_items * (t + 1) / nthreads;
            for (long i = lo; i < hi; ++i) {
                clref::g_global_id = i;
                clref::MCLightPropagation(numTriangles, factor, vStart, vStartOcc, pStart, chance,
                                          w_threshold, fetalTissueID, SurfFetalTransRxyG, rz, dimsXYZ,
                                          e_P0XYZ, gridDims, triangles, normals, mediumIDs, nMuasG, st, ix);
            }
        });
    }
    for (auto &x : th) x.join();
    return 0;
}

/* FindTriangleInPath of the reference (MCLightPropagation.cl:1037-1093). */
int clref_find_triangle(int numTriangles, float *triangles, int refTri, const float *p,
                        const float *v, float *t_out)
{
    clref::PhotonClass ph;
    ph.refTri = refTri;
    int id = ph.FindTriangleInPath(clref::float3(p[0], p[1], p[2]), clref::float3(v[0], v[1], v[2]),
                                   numTriangles, triangles);
    *t_out = ph.steptoboundary;
    return id;
}

/* GetFresnel of the reference (MCLightPropagation.cl:857-907). */
float clref_fresnel(float n1, float n2, float cosIn)
{
    clref::PhotonClass ph;
    return ph.GetFresnel(n1, n2, cosIn);
}

} // extern "C"
