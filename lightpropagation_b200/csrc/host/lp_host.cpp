// lp_host.cpp -- ImageData, Emitter, CalculatePropagation, Analysis and Logs.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <stdexcept>

#include "../../../include/lightprop.hpp"
#include "../../../include/lpcuda.h"

namespace lp {

// ================================================================== ImageData
ImageData::ImageData(const int ext[6], int ncomp) : ncomp_(ncomp)
{
    for (int i = 0; i < 6; ++i) ext_[i] = ext[i];
    int nx = ext_[1] - ext_[0] + 1, ny = ext_[3] - ext_[2] + 1;
    data_.assign((size_t)std::max(nx, 0) * std::max(ny, 0) * ncomp, 0.0f);
}
void ImageData::GetExtent(int ext[6]) const
{
    for (int i = 0; i < 6; ++i) ext[i] = ext_[i];
}
void ImageData::GetDimensions(int dims[3]) const
{
    dims[0] = ext_[1] - ext_[0] + 1;
    dims[1] = ext_[3] - ext_[2] + 1;
    dims[2] = 1;
}
size_t ImageData::index(int i, int j, int c) const
{
    if (i < ext_[0] || i > ext_[1] || j < ext_[2] || j > ext_[3] || c < 0 || c >= ncomp_)
        throw std::out_of_range("ImageData: index outside the extent");
    const size_t nx = (size_t)(ext_[1] - ext_[0] + 1);
    return ((size_t)(j - ext_[2]) * nx + (size_t)(i - ext_[0])) * ncomp_ + c;
}
float ImageData::GetScalarComponentAsFloat(int i, int j, int, int c) const { return data_[index(i, j, c)]; }
void ImageData::SetScalarComponentFromFloat(int i, int j, int, int c, float v) { data_[index(i, j, c)] = v; }
std::shared_ptr<ImageData> ImageData::Component(int c) const
{
    auto out = std::make_shared<ImageData>(ext_, 1);
    const size_t n = data_.size() / (size_t)ncomp_;
    for (size_t k = 0; k < n; ++k) out->data_[k] = data_[k * ncomp_ + c];
    return out;
}

// ================================================================== Emitter
namespace {
void normalize3(std::vector<float> &a)
{
    // Emitter::Normalize (Emitter.cpp:530-542), float arithmetic
    float f = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    a = {a[0] / f, a[1] / f, a[2] / f};
}
std::vector<float> cross3(const std::vector<float> &a, const std::vector<float> &b)
{
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
}  // namespace

void Emitter::basis()
{
    // CalculateEmitterModel (Emitter.cpp:311-339)
    eZ_ = heading_;
    std::vector<float> a(3, 0.0f);
    if (eZ_[2] != 0) {
        a = {1, 1, -(eZ_[0] + eZ_[1]) / eZ_[2]};
    } else if (eZ_[1] != 0) {
        a = {1, -eZ_[0] / eZ_[1], 0};
    } else if (eZ_[0] != 0) {
        a = {0, 1, 0};
    }
    normalize3(a);
    normalize3(eZ_);
    eY_ = cross3(eZ_, a);
    normalize3(eY_);
    eX_ = cross3(eY_, eZ_);
    normalize3(eX_);
}

void Emitter::GetEmittermodel(std::vector<float> &pStart, std::vector<float> &vStart, std::vector<int> &vStartOcc)
{
    // CalculatePointOfOrigin (Emitter.cpp:186-205): position = -heading * distance + p0
    pStart = {-heading_[0] * distance_ + p0_[0], -heading_[1] * distance_ + p0_[1], -heading_[2] * distance_ + p0_[2]};
    // CalculateStartVectorArray (Emitter.cpp:207-248) and RotateVector (Emitter.cpp:389-466)
    vStart.clear();
    for (float phi : angles_) {
        if (phi == 0) {
            vStart.insert(vStart.end(), heading_.begin(), heading_.end());
            continue;
        }
        if (!radians_) phi *= (float)(M_PI / 180.0);
        const float cosPhi = std::cos(phi), sinPhi = std::sqrt(1 - cosPhi * cosPhi);
        const std::vector<float> &v = heading_;
        std::vector<float> e_rot(3, 0.0f);
        if (v[2] != 0) e_rot = {1, 1, -(v[0] + v[1]) / v[2]};
        else if (v[1] != 0) e_rot = {1, -(v[0] + v[2]) / v[1], 1};
        else if (v[0] != 0) e_rot = {-(v[1] + v[2]) / v[0], 1, 1};
        normalize3(e_rot);
        std::vector<float> nx = cross3(e_rot, v), nxe = cross3(nx, e_rot);
        const float nDx = e_rot[0] * v[0] + e_rot[1] * v[1] + e_rot[2] * v[2];
        // VecAdd(a, b, c) of the reference adds c[0] to every component (Emitter.cpp:518-526)
        const float c0 = sinPhi * nx[0];
        std::vector<float> vn = {nDx * e_rot[0] + cosPhi * nxe[0] + c0, nDx * e_rot[1] + cosPhi * nxe[1] + c0,
                                 nDx * e_rot[2] + cosPhi * nxe[2] + c0};
        normalize3(vn);
        vStart.insert(vStart.end(), vn.begin(), vn.end());
    }
    // CalculateStartVectorOccurrences (Emitter.cpp:250-278)
    float sum = 0;
    for (float r : rri_) sum += r;
    vStartOcc.clear();
    int64_t s1 = 0;
    for (float r : rri_) {
        int occ = (int)(photons_ * r / sum);
        s1 += occ;
        vStartOcc.push_back(occ);
    }
    if (s1 < photons_ && !vStartOcc.empty()) vStartOcc[0] += (int)(photons_ - s1);
    basis();
}

void Emitter::GetBasisVectors(std::vector<float> &eX, std::vector<float> &eY, std::vector<float> &eZ)
{
    if (eZ_.empty()) basis();
    eX = eX_;
    eY = eY_;
    eZ = eZ_;
}

// ================================================================== CalculatePropagation
CalculatePropagation::CalculatePropagation() = default;

CalculatePropagation::~CalculatePropagation()
{
    if (ctx_) lp_destroy(ctx_);
}

int CalculatePropagation::check(int rc)
{
    if (rc != LP_OK) {
        err_ = lp_last_error(ctx_);
        if (verbose_) std::cerr << "liblpcuda: " << err_ << "\n";
        return 1;
    }
    return 0;
}

void CalculatePropagation::SetDeviceType(int device)
{
    if (device == 0) throw std::invalid_argument("SetDeviceType(0): the transport runs on the GPU only");
}

void CalculatePropagation::SetTissueProperties(const std::vector<float> &refractionInd,
                                                const std::vector<float> &absorbtionCoeffs,
                                                const std::vector<float> &anisotropies,
                                                const std::vector<float> &scatterCoeffs)
{
    // packs n, mua, mus, g per region (CalculatePropagation.cpp:427-451)
    const size_t s = refractionInd.size();
    nmuasG_.assign(4 * s, 0.0f);
    for (size_t i = 0; i < s; ++i) {
        nmuasG_[4 * i] = refractionInd[i];
        nmuasG_[4 * i + 1] = absorbtionCoeffs[i];
        nmuasG_[4 * i + 2] = scatterCoeffs[i];
        nmuasG_[4 * i + 3] = anisotropies[i];
    }
}

void CalculatePropagation::SetPOI(const std::vector<float> &p)
{
    for (int i = 0; i < 3; ++i) eP0XYZ_[i] = p[i];
}

void CalculatePropagation::SetBasisVectors(const std::vector<float> &eX, const std::vector<float> &eY,
                                           const std::vector<float> &eZ)
{
    for (int i = 0; i < 3; ++i) {
        eP0XYZ_[3 + i] = eX[i];
        eP0XYZ_[6 + i] = eY[i];
        eP0XYZ_[9 + i] = eZ[i];
    }
}

int CalculatePropagation::Init()
{
    if (!ctx_ && check(lp_create(&ctx_, device_))) return 1;
    const int64_t T = (int64_t)(triangles_.size() / 9);
    if (T == 0 || normals_.size() != (size_t)(3 * T) || triN_.size() != (size_t)(2 * T)) {
        err_ = "Init: triangles, normals and medium ids must describe the same mesh";
        return 1;
    }
    if (check(lp_set_mesh(ctx_, T, triangles_.data(), normals_.data(), triN_.data()))) return 1;
    if (check(lp_set_media(ctx_, (int32_t)(nmuasG_.size() / 4), nmuasG_.data()))) return 1;
    if (check(lp_set_source(ctx_, pStart_.data(), vStart_.data(), vStartOcc_.data(),
                            (int32_t)(vStart_.size() / 3), eP0XYZ_)))
        return 1;
    if (check(lp_set_fiber_source(ctx_, fiberR_, fiberNA_))) return 1;
    if (check(lp_set_tally_grid(ctx_, dimensions_.data(), detGrid_.data(), fetalTissueID_))) return 1;
    if (check(lp_set_params(ctx_, chance_, wth_, ppu_, seed_, compat_))) return 1;
    if (!rings_.empty()) {
        const int32_t vox_n[3] = {0, 0, 0};
        const float vox_d[3] = {1, 1, 1};
        if (check(lp_set_extra_tallies(ctx_, vox_n, vox_d, 0, 1.0f, (int32_t)(rings_.size() / 2), rings_.data())))
            return 1;
    }
    return check(lp_zero_tallies(ctx_));
}

// ------------------------------------------------------------------ TransportFunction
std::vector<double> TransportFunction::Forward(const std::vector<float> &mua, const std::vector<float> &mus,
                                               int64_t n, int64_t first)
{
    lp_ctx *ctx = cp_.Context();
    std::vector<float> table = cp_.GetTissueTable();
    const size_t R = table.size() / 4;
    if (!ctx || mua.size() != R || mus.size() != R) {
        err_ = "TransportFunction::Forward: Init() first; mua and mus need one value per region";
        return {};
    }
    for (size_t r = 0; r < R; ++r) {
        table[4 * r + 1] = mua[r];
        table[4 * r + 2] = mus[r];
    }
    lp_gradient g;
    if (lp_set_media(ctx, (int32_t)R, table.data()) || lp_forward(ctx, first, n, nullptr) ||
        lp_get_gradient(ctx, &g)) {
        err_ = lp_last_error(ctx);
        return {};
    }
    n_det_ = g.n_det;
    n_media_ = g.n_media;
    jmua_.assign(g.d_mua, g.d_mua + (size_t)n_det_ * n_media_);
    jmus_.assign(g.d_mus, g.d_mus + (size_t)n_det_ * n_media_);
    signal_se_.assign(g.signal_se, g.signal_se + n_det_);
    return std::vector<double>(g.signal, g.signal + n_det_);
}

bool TransportFunction::Backward(const std::vector<double> &grad_signal, std::vector<double> &grad_mua,
                                 std::vector<double> &grad_mus) const
{
    if ((int)grad_signal.size() != n_det_ || n_media_ == 0) {
        err_ = "TransportFunction::Backward: one upstream gradient per ring after a Forward";
        return false;
    }
    grad_mua.assign((size_t)n_media_, 0.0);
    grad_mus.assign((size_t)n_media_, 0.0);
    for (int d = 0; d < n_det_; ++d)
        for (int r = 0; r < n_media_; ++r) {
            grad_mua[r] += grad_signal[d] * jmua_[(size_t)d * n_media_ + r];
            grad_mus[r] += grad_signal[d] * jmus_[(size_t)d * n_media_ + r];
        }
    return true;
}

int CalculatePropagation::Propagation()
{
    if (!ctx_) {
        err_ = "Propagation: Init() has not succeeded";
        return 1;
    }
    if (check(lp_run(ctx_, 0, photons_))) return 1;
    lp_last_kernel_ms(ctx_, &kernel_ms_);
    lp_geometry g;
    lp_tallies t;
    if (check(lp_get_geometry(ctx_, &g)) || check(lp_get_tallies(ctx_, &t))) return 1;
    const double sc = 1.0 / LP_FIX_ONE;
    const int hx = g.dimx / 2, hy = g.dimy / 2;
    // images with the extents of InitLogVectors (CalculatePropagation.cpp:120-243)
    const int e_sft[6] = {-hx, hx, -hy, hy, 0, 0};
    sft_ = std::make_shared<ImageData>(e_sft, 3);
    for (size_t k = 0; k < sft_->data().size(); ++k) sft_->data()[k] = (float)(t.sft[k] * sc);
    const int e_rtd[6] = {0, g.dimR - 1, 0, g.dimAlpha - 1, 0, 0};
    rtd_ = std::make_shared<ImageData>(e_rtd, 3);
    for (size_t k = 0; k < rtd_->data().size(); ++k) rtd_->data()[k] = (float)(t.rtd[k] * sc);
    const int e_rz[6] = {-g.dimR, g.dimR, -g.dimz, 0, 0, 0};
    arz_ = std::make_shared<ImageData>(e_rz, 2);
    for (int cz = 0; cz < g.rz_nz; ++cz)        // depth row cz sits at image row -cz
        for (int col = 0; col < g.rz_nr; ++col)
            for (int c = 0; c < 2; ++c)
                arz_->SetScalarComponentFromFloat(col - g.dimR, -cz, 0, c,
                                                  (float)(t.rz[2 * ((size_t)cz * g.rz_nr + col) + c] * sc));
    region_.assign((size_t)t.n_region, 0.0);
    for (int64_t k = 0; k < t.n_region; ++k) region_[k] = t.region[k] * sc;
    if (showPercent_) std::cout << "\r| 100% \t" << std::endl;
    return 0;
}

void CalculatePropagation::PrintTimeSpent() const
{
    std::cout << "############# Calculation Time #############\n";
    std::cout << "Time in ms: " << kernel_ms_ << " \t| Time in s: " << kernel_ms_ / 1000.0 << std::endl;
}

void CalculatePropagation::PrintSimulationParams() const
{
    std::cout << "########### Simulation Parameter ###########\n";
    std::cout << "Device Name: CUDA device " << device_ << "\n";
    std::cout << "Number of Photons: " << photons_ << std::endl;
}

// ================================================================== Analysis
void Analysis::SetRTdxyLogs(const ImagePtr &image)
{
    // Analysis::SetRTdxyLogs (Analysis.cpp:447-463): x outer, y inner
    int ext[6];
    image->GetExtent(ext);
    surf_.clear();
    fetal_.clear();
    trans_.clear();
    for (int x = ext[0]; x <= ext[1]; x++)
        for (int y = ext[2]; y <= ext[3]; y++) {
            surf_.push_back(image->GetScalarComponentAsFloat(x, y, 0, 0));
            fetal_.push_back(image->GetScalarComponentAsFloat(x, y, 0, 1));
            trans_.push_back(image->GetScalarComponentAsFloat(x, y, 0, 2));
        }
}

void Analysis::CalculateSurfaceSums()
{
    // Analysis::CalculateSurfaceSums (Analysis.cpp:144-156), float accumulation as there
    float s = 0, t = 0, f = 0;
    for (float v : surf_) s += v;
    for (float v : trans_) t += v;
    for (float v : fetal_) f += v;
    surf_sum_ = s;
    trans_sum_ = t;
    fetal_sum_ = f;
}

void Analysis::PrintAnalysis() const
{
    // Analysis::PrintAnalysis / PrintSurfaceSums (Analysis.cpp:529-545)
    std::cout << "################ Analysis ##################\n";
    std::cout << "Number of Photons: " << photons_ << "\n";
    std::cout << "SurfRxy: " << surf_sum_ << " | in %: " << surf_sum_ / photons_ * 100 << "\n";
    std::cout << "TransRxy: " << trans_sum_ << " | in %: " << trans_sum_ / photons_ * 100 << "\n";
    std::cout << "FetalRxy: " << fetal_sum_ << " | in %: " << fetal_sum_ / photons_ * 100 << "\n";
    std::cout << "Surf+TransRxy: " << surf_sum_ + trans_sum_ << "\n";
    std::cout << "############################################" << std::endl;
}

// ================================================================== Logs
std::string Logs::out_name(const std::string &fname, const char *suffix) const
{
    return dir_ + fname.substr(0, fname.find_last_of('.')) + suffix;
}

float Logs::ScalePerRadius1D(int ir) const
{
    // Logs::ScalePerRadius1D (Logs.cpp:651-659): 1 / ((ir + 0.5) * 2 pi dr^2 N)
    double dr = grid_[3];
    float scale1 = (float)(2.0 * M_PI * dr * dr * (double)photons_);
    return (float)(1.0 / ((ir + 0.5) * scale1));
}

float Logs::ScalePerAngle1D(int ia) const
{
    // Logs::ScalePerAngle1D (Logs.cpp:661-672): 1 / (sin((ia + 0.5) da) 2 pi da N)
    double da = grid_[5] * M_PI / 180;
    float scale1 = (float)(2.0 * M_PI * da * (double)photons_);
    return (float)(1.0 / (std::sin((ia + 0.5) * da) * scale1));
}

float Logs::Scale2D(int ir, int ia) const
{
    // Logs::Scale2D (Logs.cpp:493-516)
    double dr = grid_[3];
    double da = grid_[5] * M_PI / 180;
    float scale1 = (float)(4.0 * M_PI * M_PI * dr * std::sin(da / 2) * dr * (double)photons_);
    return (float)(1.0 / ((ir + 0.5) * std::sin(2.0 * (ia + 0.5) * da) * scale1));
}

void Logs::SaveSurfaceArr(const std::string &fname, const ImagePtr &image) const
{
    std::ofstream f(dir_ + fname);
    int ext[6];
    image->GetExtent(ext);
    for (int n = ext[2]; n <= ext[3]; n++) {
        for (int m = ext[0]; m <= ext[1]; m++) f << image->GetScalarComponentAsFloat(m, n, 0, 0) << "\t";
        f << "\n";
    }
}

void Logs::SaveRecordRd(const std::string &fname, const ImagePtr &image) const
{
    std::ofstream f(out_name(fname, "_Rd.txt"));
    int ext[6];
    image->GetExtent(ext);
    for (int n = ext[2]; n <= ext[3]; n++) {
        for (int m = ext[0]; m <= ext[1]; m++) f << image->GetScalarComponentAsFloat(m, n, 0, 0) * Scale2D(m, n) << "\t";
        f << "\n";
    }
}

void Logs::CalcReflectancePerRadius(const std::string &fname, const ImagePtr &image) const
{
    std::ofstream f(out_name(fname, "_perRadius.txt"));
    int ext[6];
    image->GetExtent(ext);
    for (int r = ext[0]; r <= ext[1]; r++) {
        float refl = 0;
        for (int a = ext[2]; a <= ext[3]; a++) refl += image->GetScalarComponentAsFloat(r, a, 0, 0);
        f << r * grid_[3] << "\t" << refl * ScalePerRadius1D(std::abs(r)) << "\n";
    }
}

void Logs::CalcReflectancePerAngle(const std::string &fname, const ImagePtr &image) const
{
    std::ofstream f(out_name(fname, "_perAngle.txt"));
    int ext[6];
    image->GetExtent(ext);
    for (int n = ext[2]; n <= ext[3]; n++) {
        float refl = 0;
        for (int m = ext[0]; m <= ext[1]; m++) refl += image->GetScalarComponentAsFloat(m, n, 0, 0);
        f << n * grid_[5] << "\t" << refl * ScalePerAngle1D(n) << "\n";
    }
}

void Logs::FluenceZ(const std::string &fname, const ImagePtr &fluence) const
{
    std::ofstream f(out_name(fname, "_perZ.txt"));
    int ext[6];
    fluence->GetExtent(ext);
    for (int z = ext[2]; z <= ext[3]; z++) {
        float fl = 0;
        for (int r = ext[0]; r <= ext[1]; r++) fl += fluence->GetScalarComponentAsFloat(r, z, 0, 0);
        f << std::abs(z) * grid_[2] << "\t" << fl / (grid_[2] * photons_) << "\n";
    }
}

}  // namespace lp
