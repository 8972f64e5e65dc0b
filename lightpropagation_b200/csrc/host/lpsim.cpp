// lpsim.cpp -- command-line driver with the flow of the reference's main
// (src/main/main.cpp:64-347): import config + mesh, build the emitter, simulate,
// analyse, write the text logs.  The VTK render window (-g) and PNG pictures are
// not provided (no graphics stack).
//
//   lpsim -f config.xml [-s] [-a] [-t] [-v] [-n photons] [--seed S] [--compat C]
//         [--exact] [-o outdir] [--device D]
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>

#include "../../../include/lightprop.hpp"
#include "../../../include/lpcuda.h"

int main(int argc, char **argv)
{
    std::string cfgpath, outdir;
    bool sim = false, analyse = false, timing = false, verbose = false, exact = false, have_out = false;
    long long photons = -1;
    unsigned long long seed = 0x4C50;
    unsigned compat = 7;
    int device = 0;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto next = [&](const char *what) -> const char * {
            if (i + 1 >= argc) {
                std::cerr << "lpsim: " << what << " needs a value\n";
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "-f") cfgpath = next("-f");
        else if (a == "-s") sim = true;
        else if (a == "-a") analyse = true;
        else if (a == "-t") timing = true;
        else if (a == "-v") verbose = true;
        else if (a == "-n") photons = std::atoll(next("-n"));
        else if (a == "--seed") seed = std::strtoull(next("--seed"), nullptr, 0);
        else if (a == "--compat") compat = (unsigned)std::strtoul(next("--compat"), nullptr, 0);
        else if (a == "--exact") exact = true;
        else if (a == "--device") device = std::atoi(next("--device"));
        else if (a == "-o") { outdir = next("-o"); have_out = true; }
        else {
            std::cerr << "usage: lpsim -f config.xml [-s] [-a] [-t] [-v] [-n photons] [--seed S] [--compat C] "
                         "[--exact] [-o outdir] [--device D]\n";
            return 2;
        }
    }
    if (cfgpath.empty()) {
        std::cerr << "lpsim: -f config.xml is required\n";
        return 2;
    }
    try {
        lp::Config c = lp::ReadConfig(cfgpath);
        std::vector<std::string> names;
        std::vector<float> n, mua, g, mus;
        for (const auto &t : c.tissues) {
            names.push_back(t.name);
            n.push_back(t.n);
            mua.push_back(t.mua);
            g.push_back(t.g);
            mus.push_back(t.mus);
        }
        lp::Mesh mesh = lp::ReadObj(c.modelfile, names);
        std::vector<float> angles, rri;
        lp::ReadEmitterFile(c.emitterfile, angles, rri);
        if (photons > 0) c.numberOfPhotons = photons;
        lp::Emitter em;
        em.SetNumberOfPhotons(c.numberOfPhotons);
        em.SetPointInPlane({c.emitter_pos[0], c.emitter_pos[1], c.emitter_pos[2]});
        em.SetDistanceToSurface(c.emitter_distance);
        em.SetRadiationCharacteristics(angles, rri);
        em.SetEmitterHeading({c.emitter_heading[0], c.emitter_heading[1], c.emitter_heading[2]});
        std::vector<float> pStart, vStart, eX, eY, eZ;
        std::vector<int> occ;
        em.GetEmittermodel(pStart, vStart, occ);
        em.GetBasisVectors(eX, eY, eZ);
        if (verbose)
            std::cout << "model " << c.modelfile << ": " << mesh.n_tri() << " triangles, " << names.size()
                      << " regions\n";
        if (!sim) return 0;
        lp::CalculatePropagation cp;
        cp.SetVerbosity(verbose);
        cp.SetDevice(device);
        cp.SetTissueProperties(n, mua, g, mus);
        cp.SetFetalTissueID(c.fetalID);
        cp.SetDimensions({c.dims[0], c.dims[1], c.dims[2]});
        cp.SetDetectionGridDimensions(std::vector<float>(c.detGrid, c.detGrid + 6));
        cp.SetTriangles(mesh.tri);
        cp.SetNormals(mesh.nrm);
        cp.SetInnerAndOuterTissueIndices(mesh.med);
        cp.SetPixelPerUnitFactor(c.ppu);
        cp.SetStartTrajectories(vStart, occ);
        cp.SetStartPoint(pStart);
        cp.SetPOI({c.emitter_pos[0], c.emitter_pos[1], c.emitter_pos[2]});
        cp.SetBasisVectors(eX, eY, eZ);
        cp.SetChanceForRoulette(c.chance);
        cp.SetWeightThreshold(c.weightThreshold);
        cp.SetNumberOfPhotons(c.numberOfPhotons);
        cp.SetSeed(seed);
        cp.SetCompat(compat);
        if (cp.Init() != 0) {
            std::cerr << "lpsim: Init failed: " << cp.LastError() << "\n";
            return 1;
        }
        if (exact && lp_set_arithmetic(cp.Context(), 1) != 0) return 1;
        if (timing) cp.PrintSimulationParams();
        if (cp.Propagation() != 0) {
            std::cerr << "lpsim: Propagation failed: " << cp.LastError() << "\n";
            return 1;
        }
        if (timing) cp.PrintTimeSpent();
        if (analyse) {
            lp::Analysis an;
            an.SetNumberOfPhotons(c.numberOfPhotons);
            an.SetRTdxyLogs(cp.GetSFTImage());
            an.CalculateSurfaceSums();
            an.PrintAnalysis();
            if (c.saveLogFiles || have_out) {
                std::string dir = have_out ? outdir : c.saveDir;
                if (!dir.empty() && dir.back() != '/') dir += '/';
                std::cout << "Writing Files in " << dir << "\n" << std::endl;
                lp::Logs log;
                log.SetSaveDir(dir);
                log.SetGridDimensions(std::vector<float>(c.detGrid, c.detGrid + 6));
                log.SetNumberOfPhotons(c.numberOfPhotons);
                const std::string sf = c.surfaceFilename.empty() ? "SurfRxy.txt" : c.surfaceFilename;
                const std::string tf = c.transmissionFilename.empty() ? "TransRxy.txt" : c.transmissionFilename;
                const std::string ff = c.fetalFilename.empty() ? "FetalRxy.txt" : c.fetalFilename;
                const std::string az = c.absorbYZFilename.empty() ? "FluencePrz.txt" : c.absorbYZFilename;
                log.SaveSurfaceArr(sf, cp.GetSFTImage(lp::Rxy_Log_SURF));
                log.SaveRecordRd(sf, cp.GetRTdImage(lp::Rxy_Log_SURF));
                log.CalcReflectancePerRadius(sf, cp.GetRTdImage(lp::Rxy_Log_SURF));
                log.CalcReflectancePerAngle(sf, cp.GetRTdImage(lp::Rxy_Log_SURF));
                log.CalcReflectancePerRadius(tf, cp.GetRTdImage(lp::Rxy_Log_TRANS));
                log.CalcReflectancePerAngle(tf, cp.GetRTdImage(lp::Rxy_Log_TRANS));
                log.CalcReflectancePerRadius(ff, cp.GetRTdImage(lp::Rxy_Log_FETAL));
                log.CalcReflectancePerAngle(ff, cp.GetRTdImage(lp::Rxy_Log_FETAL));
                log.FluenceZ(az, cp.GetPhirzImage());
                std::cout << "Writing Done." << std::endl;
            }
        }
    } catch (const std::exception &e) {
        std::cerr << "lpsim: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
