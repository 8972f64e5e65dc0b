// lph_capi.cpp -- C entry points of the host layer (liblphost.so) for callers that
// cannot use C++ (the Python package and its tests): load a reference-format model
// (config XML + OBJ + emitter file) into the arrays lp_set_* expect.
#include <cstring>
#include <stdexcept>

#include "../../../include/lightprop.hpp"

struct lph_model {
    lp::Config cfg;
    lp::Mesh mesh;
    std::vector<float> nmuasg;
    float p_start[3], v_start[3], ep0xyz[12];
};

extern "C" {

lph_model *lph_load(const char *config_path, char *err, int errlen)
{
    try {
        auto *m = new lph_model;
        m->cfg = lp::ReadConfig(config_path);
        std::vector<std::string> names;
        for (const auto &t : m->cfg.tissues) {
            names.push_back(t.name);
            m->nmuasg.insert(m->nmuasg.end(), {t.n, t.mua, t.mus, t.g});
        }
        m->mesh = lp::ReadObj(m->cfg.modelfile, names);
        std::vector<float> angles, rri;
        lp::ReadEmitterFile(m->cfg.emitterfile, angles, rri);
        lp::Emitter em;
        em.SetNumberOfPhotons(m->cfg.numberOfPhotons);
        em.SetPointInPlane({m->cfg.emitter_pos[0], m->cfg.emitter_pos[1], m->cfg.emitter_pos[2]});
        em.SetDistanceToSurface(m->cfg.emitter_distance);
        em.SetRadiationCharacteristics(angles, rri);
        em.SetEmitterHeading({m->cfg.emitter_heading[0], m->cfg.emitter_heading[1], m->cfg.emitter_heading[2]});
        std::vector<float> p, v, eX, eY, eZ;
        std::vector<int> occ;
        em.GetEmittermodel(p, v, occ);
        em.GetBasisVectors(eX, eY, eZ);
        for (int i = 0; i < 3; ++i) {
            m->p_start[i] = p[i];
            m->v_start[i] = v[i];
            m->ep0xyz[i] = m->cfg.emitter_pos[i];
            m->ep0xyz[3 + i] = eX[i];
            m->ep0xyz[6 + i] = eY[i];
            m->ep0xyz[9 + i] = eZ[i];
        }
        return m;
    } catch (const std::exception &e) {
        if (err && errlen > 0) {
            std::strncpy(err, e.what(), (size_t)errlen - 1);
            err[errlen - 1] = 0;
        }
        return nullptr;
    }
}

void lph_free(lph_model *m) { delete m; }
int64_t lph_n_tri(const lph_model *m) { return m->mesh.n_tri(); }
const float *lph_tri(const lph_model *m) { return m->mesh.tri.data(); }
const float *lph_nrm(const lph_model *m) { return m->mesh.nrm.data(); }
const float *lph_vn(const lph_model *m) { return m->mesh.vn.data(); }
const int32_t *lph_med(const lph_model *m) { return m->mesh.med.data(); }
int32_t lph_n_media(const lph_model *m) { return (int32_t)(m->nmuasg.size() / 4); }
const float *lph_nmuasg(const lph_model *m) { return m->nmuasg.data(); }

void lph_source(const lph_model *m, float *p_start, float *v_start, float *ep0xyz)
{
    std::memcpy(p_start, m->p_start, 12);
    std::memcpy(v_start, m->v_start, 12);
    std::memcpy(ep0xyz, m->ep0xyz, 48);
}

// Write one reference-format log (lp::Logs) of an image with extent ext and ncomp
// components, values ordered x fastest then y (component innermost), as lp::ImageData
// stores them.  kind: 0 SaveSurfaceArr, 1 SaveRecordRd, 2 CalcReflectancePerRadius,
// 3 CalcReflectancePerAngle, 4 FluenceZ.  Returns 0, or 1 for an unknown kind.
int lph_write_log(const char *dir, const char *fname, int kind, const float *values, const int32_t *ext, int ncomp,
                  const float *grid, int64_t photons)
{
    const int e[6] = {ext[0], ext[1], ext[2], ext[3], ext[4], ext[5]};
    auto img = std::make_shared<lp::ImageData>(e, ncomp);
    std::memcpy(img->data().data(), values, img->data().size() * sizeof(float));
    lp::Logs logs;
    logs.SetSaveDir(dir);
    logs.SetGridDimensions(std::vector<float>(grid, grid + 6));
    logs.SetNumberOfPhotons(photons);
    switch (kind) {
    case 0: logs.SaveSurfaceArr(fname, img); return 0;
    case 1: logs.SaveRecordRd(fname, img); return 0;
    case 2: logs.CalcReflectancePerRadius(fname, img); return 0;
    case 3: logs.CalcReflectancePerAngle(fname, img); return 0;
    case 4: logs.FluenceZ(fname, img); return 0;
    default: return 1;
    }
}

// lp::Analysis surface sums of an SFT image (3 components): surf, fetal, trans.
void lph_surface_sums(const float *values, const int32_t *ext, double *out)
{
    const int e[6] = {ext[0], ext[1], ext[2], ext[3], ext[4], ext[5]};
    auto img = std::make_shared<lp::ImageData>(e, 3);
    std::memcpy(img->data().data(), values, img->data().size() * sizeof(float));
    lp::Analysis a;
    a.SetRTdxyLogs(img);
    a.CalculateSurfaceSums();
    out[0] = a.SurfaceSum();
    out[1] = a.FetalSum();
    out[2] = a.TransSum();
}

void lph_grid(const lph_model *m, float *dims, float *det_grid, int32_t *fetal_id, float *chance, float *w_th,
              float *ppu, int64_t *photons)
{
    std::memcpy(dims, m->cfg.dims, 12);
    std::memcpy(det_grid, m->cfg.detGrid, 24);
    *fetal_id = m->cfg.fetalID;
    *chance = m->cfg.chance;
    *w_th = m->cfg.weightThreshold;
    *ppu = m->cfg.ppu;
    *photons = m->cfg.numberOfPhotons;
}

}  // extern "C"
