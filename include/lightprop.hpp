// lightprop.hpp -- C++ host layer of the B200 transport library (liblphost.so).
//
// Mirrors the reference's host classes around the hot path without VTK:
//   ReadXML / ImportExport   src/IO/ReadXML.cpp, src/IO/ImportExport.cpp  (config + OBJ mesh, region ids)
//   Emitter                  src/Model/Emitter.cpp                         (source geometry)
//   CalculatePropagation     src/Simulation/CalculatePropagation.hpp:212-388 (launcher; forwards to lpcuda.h)
//   Analysis                 src/Analysis/Analysis.cpp:144-156, 447-538    (surface sums)
//   Logs                     src/IO/Logs.cpp:337-561, 651-713, 1075-1110   (text outputs)
// VTK types are replaced by ImageData (extent + float components) and plain vectors.
#pragma once
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

struct lp_ctx;

namespace lp {

// ------------------------------------------------------------------ images
// Minimal vtkImageData: 2-D extent [x0,x1] x [y0,y1] (z fixed 0) with ncomp float components.
class ImageData {
public:
    ImageData() = default;
    ImageData(const int ext[6], int ncomp);
    void GetExtent(int ext[6]) const;
    void GetDimensions(int dims[3]) const;
    int GetNumberOfScalarComponents() const { return ncomp_; }
    float GetScalarComponentAsFloat(int i, int j, int k, int c) const;
    void SetScalarComponentFromFloat(int i, int j, int k, int c, float v);
    std::vector<float> &data() { return data_; }
    const std::vector<float> &data() const { return data_; }
    std::shared_ptr<ImageData> Component(int c) const;

private:
    int ext_[6] = {0, -1, 0, -1, 0, 0};
    int ncomp_ = 0;
    std::vector<float> data_;
    size_t index(int i, int j, int c) const;
};
using ImagePtr = std::shared_ptr<ImageData>;

// ------------------------------------------------------------------ config
struct Tissue {
    int id = 0;
    std::string name;
    float n = 1, mua = 0, mus = 0, g = 0;
};

// Keys of the reference's <config> XML (ReadXML::ExtractConfigVars, ReadXML.cpp:109-168).
struct Config {
    std::string modelfile, emitterfile, saveDir;
    float ppu = 1;                       // PixelPerUnit
    float dims[3] = {1, 1, 1};           // model/dimensions
    std::vector<Tissue> tissues;         // tissueList, indexed by ID
    float emitter_pos[3] = {0, 0, 0};
    float emitter_distance = 0;
    float emitter_heading[3] = {0, 0, 1};
    int64_t numberOfPhotons = 1;
    int numPhotonsInteractions = 100;
    float chance = 0.1f, weightThreshold = 1e-4f;
    bool saveLogFiles = false;
    int fetalID = 1;
    float detGrid[6] = {1, 1, 1, 1, 1, 1};   // x y z r phi rho
    std::string surfaceFilename, fetalFilename, transmissionFilename, absorbXZFilename, absorbYZFilename;
    std::string scale, coordsystem, colormap;
    std::vector<std::string> surfNames;      // analyse/boundaries/surfName
};
// Parses the config file; relative or missing model/emitter paths are resolved
// against the config file's directory.  Throws std::runtime_error on failure.
Config ReadConfig(const std::string &path);

// ------------------------------------------------------------------ mesh
struct Mesh {
    std::vector<float> tri;   // 9 floats per triangle (K, L, M)
    std::vector<float> nrm;   // 3 floats per triangle, unit (B-A)x(C-A)
    std::vector<int32_t> med; // inner, outer region per triangle
    std::vector<float> vn;    // 3 floats per triangle: the file's first vn of the face (0 if none)
    std::vector<int32_t> surface_ids;      // triangles of named surfaces (g <id>_<name>)
    std::vector<std::string> surface_names;
    int64_t n_tri() const { return (int64_t)(tri.size() / 9); }
};
// Wavefront OBJ as vtkOBJReader + GenMediumIDsFromObjModel read it
// (ImportExport.cpp:341-392, 952-1053): `o <name>` sets the inner region to the
// index of <name> in `tissue_names`, `g <id>` / `g <id>_<surf>` set the outer region,
// every `f` line is one cell whose first three vertices form the triangle.
Mesh ReadObj(const std::string &path, const std::vector<std::string> &tissue_names);

// Emitter directions file: lines "<angle> <relative intensity>" (ImportExport.cpp:393-433).
void ReadEmitterFile(const std::string &path, std::vector<float> &angles, std::vector<float> &rri);

// ------------------------------------------------------------------ emitter
// Source geometry of Emitter::CalculateEmitterModel (Emitter.cpp:186-339), float arithmetic.
class Emitter {
public:
    void SetNumberOfPhotons(int64_t n) { photons_ = n; }
    void SetPointInPlane(const std::vector<float> &p) { p0_ = p; }
    void SetDistanceToSurface(float d) { distance_ = d; }
    void SetRadiationCharacteristics(const std::vector<float> &angles, const std::vector<float> &rri)
    {
        angles_ = angles;
        rri_ = rri;
    }
    void SetEmitterHeading(const std::vector<float> &h) { heading_ = h; }
    void AngleIsDegree() { radians_ = false; }
    void GetEmittermodel(std::vector<float> &pStart, std::vector<float> &vStart, std::vector<int> &vStartOcc);
    void GetBasisVectors(std::vector<float> &eX, std::vector<float> &eY, std::vector<float> &eZ);

private:
    int64_t photons_ = 1;
    float distance_ = 1;
    bool radians_ = true;
    std::vector<float> p0_{0, 0, 0}, heading_{0, 0, 1}, angles_{0}, rri_{1};
    std::vector<float> eX_, eY_, eZ_;
    void basis();
};

// ------------------------------------------------------------------ launcher
enum { Rxy_Log_SURF = 0, Rxy_Log_FETAL = 1, Rxy_Log_TRANS = 2 };

class CalculatePropagation {
public:
    CalculatePropagation();
    ~CalculatePropagation();
    CalculatePropagation(const CalculatePropagation &) = delete;
    CalculatePropagation &operator=(const CalculatePropagation &) = delete;

    void SetVerbosity(bool v) { verbose_ = v; }
    void SetShowPercentDone(bool s) { showPercent_ = s; }
    void SetDeviceType(int device);   // 0 = CPU is rejected: the product path is CUDA only
    void SetDevice(int cuda_device) { device_ = cuda_device; }
    void SetTissueProperties(const std::vector<float> &refractionInd, const std::vector<float> &absorbtionCoeffs,
                             const std::vector<float> &anisotropies, const std::vector<float> &scatterCoeffs);
    void SetFetalTissueID(int id) { fetalTissueID_ = id; }
    void SetDimensions(const std::vector<float> &dims) { dimensions_ = dims; }
    void SetDetectionGridDimensions(const std::vector<float> &g) { detGrid_ = g; }
    void SetDetectionGridDimensions(float x, float y, float z, float r, float phi, float rho)
    {
        detGrid_ = {x, y, z, r, phi, rho};
    }
    void SetTriangles(const std::vector<float> &tri9) { triangles_ = tri9; }
    void SetNormals(const std::vector<float> &nrm3) { normals_ = nrm3; }
    void SetInnerAndOuterTissueIndices(const std::vector<int32_t> &med2) { triN_ = med2; }
    void SetPixelPerUnitFactor(float f) { ppu_ = f; }
    void SetStartTrajectories(const std::vector<float> &traj, const std::vector<int> &occ)
    {
        vStart_ = traj;
        vStartOcc_ = occ;
    }
    void SetStartPoint(const std::vector<float> &p) { pStart_ = p; }
    void SetPOI(const std::vector<float> &p);
    void SetBasisVectors(const std::vector<float> &eX, const std::vector<float> &eY, const std::vector<float> &eZ);
    void SetChanceForRoulette(float c) { chance_ = c; }
    void SetWeightThreshold(float w) { wth_ = w; }
    void SetNumberOfPhotons(int64_t n) { photons_ = n; }
    void SetNumberOfPhotonInteractions(int n) { interactions_ = n; }
    void SetSeed(uint64_t s) { seed_ = s; }
    void SetCompat(uint32_t c) { compat_ = c; }
    void SetFiberSource(float radius, float na) { fiberR_ = radius; fiberNA_ = na; }
    // ring detectors (no reference counterpart): [inner, outer) radii in the emitter
    // plane, two floats per ring; surface exits inside a ring are scored there
    void SetRingDetectors(const std::vector<float> &radii) { rings_ = radii; }
    const std::vector<float> &GetTissueTable() const { return nmuasG_; }   // n, mua, mus, g per region

    int64_t GetNumberOfPhotons() const { return photons_; }
    float GetChanceForRoulette() const { return chance_; }
    float GetWeightThreshold() const { return wth_; }

    int Init();          // returns 0 (SUCCESS) or 1 (FAILURE)
    int Propagation();   // returns 0 (SUCCESS) or 1 (FAILURE)

    ImagePtr GetSFTImage() const { return sft_; }
    ImagePtr GetSFTImage(int component) const { return sft_ ? sft_->Component(component) : nullptr; }
    ImagePtr GetRTdImage() const { return rtd_; }
    ImagePtr GetRTdImage(int component) const { return rtd_ ? rtd_->Component(component) : nullptr; }
    ImagePtr GetArzImage() const { return arz_ ? arz_->Component(0) : nullptr; }
    ImagePtr GetPhirzImage() const { return arz_ ? arz_->Component(1) : nullptr; }
    const std::vector<double> &GetRegionAbsorption() const { return region_; }

    void PrintTimeSpent() const;
    void PrintSimulationParams() const;
    const std::string &LastError() const { return err_; }
    lp_ctx *Context() { return ctx_; }

private:
    lp_ctx *ctx_ = nullptr;
    int device_ = 0;
    bool verbose_ = false, showPercent_ = false;
    std::vector<float> nmuasG_, dimensions_{1, 1, 1}, detGrid_{1, 1, 1, 1, 1, 1};
    std::vector<float> triangles_, normals_, vStart_{0, 0, 1}, pStart_{0, 0, 0};
    std::vector<int32_t> triN_;
    std::vector<int> vStartOcc_{1};
    float eP0XYZ_[12] = {0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1};
    int fetalTissueID_ = 1, interactions_ = 100;
    float ppu_ = 100, chance_ = 0.5f, wth_ = 0.001f, fiberR_ = 0, fiberNA_ = 0;
    std::vector<float> rings_;
    int64_t photons_ = 1;
    uint64_t seed_ = 0x4C50;
    uint32_t compat_ = 7;
    float kernel_ms_ = 0;
    ImagePtr sft_, rtd_, arz_;
    std::vector<double> region_;
    std::string err_;
    int check(int rc);
};

// ------------------------------------------------------------------ differentiation
// Ring-detector signals S_d as a function of every region's absorption and scattering
// coefficients, shaped like an autograd Function: Forward traces photons with the
// adjoint path-length / interaction sums on (lp_forward) and keeps the Jacobians,
// Backward returns the vector-Jacobian product.  Mesh, source and rings come from an
// initialised CalculatePropagation.  No reference counterpart.
class TransportFunction {
public:
    explicit TransportFunction(CalculatePropagation &cp) : cp_(cp) {}
    // S_d for photons [first, first + n) with mua[r], mus[r] replacing the regions'
    // coefficients (n and g unchanged); empty on failure (see LastError)
    std::vector<double> Forward(const std::vector<float> &mua, const std::vector<float> &mus, int64_t n,
                                int64_t first = 0);
    // grad_mua[r] = sum_d grad_signal[d] dS_d/dmua_r, grad_mus likewise; false on failure
    bool Backward(const std::vector<double> &grad_signal, std::vector<double> &grad_mua,
                  std::vector<double> &grad_mus) const;
    const std::vector<double> &JacobianMua() const { return jmua_; }   // [n_det][n_media]
    const std::vector<double> &JacobianMus() const { return jmus_; }
    const std::vector<double> &SignalError() const { return signal_se_; }
    const std::string &LastError() const { return err_; }

private:
    CalculatePropagation &cp_;
    std::vector<double> jmua_, jmus_, signal_se_;
    int n_det_ = 0, n_media_ = 0;
    mutable std::string err_;
};

// ------------------------------------------------------------------ analysis
class Analysis {
public:
    void SetNumberOfPhotons(int64_t n) { photons_ = n; }
    void SetRTdxyLogs(const ImagePtr &sft);   // Analysis.cpp:447-463
    void CalculateSurfaceSums();               // Analysis.cpp:144-156
    void PrintAnalysis() const;                // Analysis.cpp:529-545
    double SurfaceSum() const { return surf_sum_; }
    double FetalSum() const { return fetal_sum_; }
    double TransSum() const { return trans_sum_; }

private:
    int64_t photons_ = 1;
    std::vector<float> surf_, fetal_, trans_;
    double surf_sum_ = 0, fetal_sum_ = 0, trans_sum_ = 0;
};

// ------------------------------------------------------------------ logs
class Logs {
public:
    void SetSaveDir(const std::string &d) { dir_ = d; }
    void SetGridDimensions(const std::vector<float> &g) { grid_ = g; }
    void SetNumberOfPhotons(int64_t n) { photons_ = n; }
    void SaveSurfaceArr(const std::string &fname, const ImagePtr &img) const;          // Logs.cpp:337-362
    void SaveRecordRd(const std::string &fname, const ImagePtr &img) const;            // Logs.cpp:368-402
    void CalcReflectancePerRadius(const std::string &fname, const ImagePtr &img) const;  // Logs.cpp:521-561
    void CalcReflectancePerAngle(const std::string &fname, const ImagePtr &img) const;   // Logs.cpp:674-713
    void FluenceZ(const std::string &fname, const ImagePtr &phirz) const;                // Logs.cpp:1075-1110
    float Scale2D(int ir, int ia) const;
    float ScalePerRadius1D(int ir) const;
    float ScalePerAngle1D(int ia) const;

private:
    std::string dir_;
    std::vector<float> grid_{1, 1, 1, 1, 1, 1};
    int64_t photons_ = 1;
    std::string out_name(const std::string &fname, const char *suffix) const;
};

}  // namespace lp
