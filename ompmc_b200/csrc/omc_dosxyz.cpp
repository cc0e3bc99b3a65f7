// The omc_dosxyz program as a library call: `.inp` in, `.3ddose` out
// (omc_dosxyz.c:1072-1307).  Host-only; drives the engine through the C ABI.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "omc_host.h"
#include "../../include/omcgpu.h"

using namespace omc;

namespace {

int fail(int code, const std::string &msg) {
    std::fprintf(stderr, "omc_dosxyz: %s\n", msg.c_str());
    return code;
}

bool need(const Input &in, const char *key, std::string &v) { return in.get(key, v); }

// `.3ddose`: dims, boundaries, dose (%e), relative uncertainty (%f), x
// fastest (outputResults, omc_dosxyz.c:801-886).
int write_3ddose(const std::string &path, const Phantom &ph, const std::vector<double> &dose,
                 const std::vector<double> &unc) {
    FILE *f = std::fopen(path.c_str(), "w");
    if (!f) return fail(OMC_E_IO, "unable to open output file " + path);
    std::fprintf(f, "%5d%5d%5d\n", ph.nx, ph.ny, ph.nz);
    for (auto *b : {&ph.xb, &ph.yb, &ph.zb}) {
        for (double v : *b) std::fprintf(f, "%f ", v);
        std::fprintf(f, "\n");
    }
    for (double v : dose) std::fprintf(f, "%e ", v);
    std::fprintf(f, "\n");
    for (double v : unc) std::fprintf(f, "%f ", v);
    std::fprintf(f, "\n");
    std::fclose(f);
    return OMC_OK;
}

}  // namespace

extern "C" int omc_dosxyz_run(const char *inp_base, const char *out_name, int mode, int verbose) {
    if (!inp_base || !out_name) return fail(OMC_E_ARG, "input and output names are required");
    Input in;
    std::string err, v;
    int rc = in.parse_file(std::string(inp_base) + ".inp", err);
    if (rc) return fail(rc, err);

    Phantom ph;
    if (!need(in, "phantom file", v)) return fail(OMC_E_ARG, "Can not find 'phantom file' key on input file.");
    if ((rc = read_egsphant(strip_spaces(v), ph, err))) return fail(rc, err);

    std::string pegs, pgs4, data, outdir;
    if (!need(in, "pegs file", pegs)) return fail(OMC_E_ARG, "Can not find 'pegs file' key on input file.");
    if (!need(in, "pgs4form file", pgs4)) return fail(OMC_E_ARG, "Can not find 'pgs4form file' key on input file.");
    if (!need(in, "data folder", data)) return fail(OMC_E_ARG, "Can not find 'data folder' key on input file.");
    if (!need(in, "output folder", outdir)) return fail(OMC_E_ARG, "Can not find 'output folder' key on input file.");
    std::vector<const char *> media;
    for (auto &m : ph.media) media.push_back(m.c_str());
    omc_tables *tab = nullptr;
    pegs = strip_spaces(pegs);
    pgs4 = strip_spaces(pgs4);
    data = strip_spaces(data);
    if ((rc = omc_tables_build(pegs.c_str(), pgs4.c_str(), data.c_str(), media.data(), (int)media.size(), &tab)))
        return fail(rc, omc_last_error());
    // the table set is released on every return below
    std::unique_ptr<omc_tables, void (*)(omc_tables *)> tab_guard(tab, omc_tables_free);

    omc_options opt;
    omc_options_default(&opt);
    if (!need(in, "global ecut", v)) return fail(OMC_E_ARG, "Can not find 'global ecut' key on input file.");
    opt.ecut = std::atof(v.c_str());
    if (!need(in, "global pcut", v)) return fail(OMC_E_ARG, "Can not find 'global pcut' key on input file.");
    opt.pcut = std::atof(v.c_str());
    if (!need(in, "nsplit", v)) return fail(OMC_E_ARG, "Can not find 'nsplit' key on input file.");
    opt.nsplit = std::atoi(v.c_str());
    if (opt.nsplit > 1 && verbose) std::printf("Photon splitting enabled, nsplit = %d\n", opt.nsplit);

    // source (initSource, omc_dosxyz.c:337-632)
    omc_beam beam{};
    std::vector<double> cdf1(1000), cdf2(1000);
    if (in.get("spectrum file", v)) {
        int n = 0;
        if ((rc = omc_spectrum_load(strip_spaces(v).c_str(), cdf1.data(), cdf2.data(), &n))) {
            return fail(rc, omc_last_error());
        }
        beam.energy.n = n;
        beam.energy.cdf1 = cdf1.data();
        beam.energy.cdf2 = cdf2.data();
    } else {
        if (!need(in, "mono energy", v)) {
            return fail(OMC_E_ARG, "Can not find 'mono energy' key on input file.");
        }
        beam.energy.mono_energy = std::atof(v.c_str());
    }
    if (!need(in, "collimator bounds", v) ||
        std::sscanf(v.c_str(), "%lf %lf %lf %lf", &beam.xinl, &beam.xinu, &beam.yinl, &beam.yinu) != 4) {
        return fail(OMC_E_ARG, "Can not find 'collimator bounds' key on input file.");
    }
    if (!need(in, "charge", v)) {
        return fail(OMC_E_ARG, "Can not find 'charge' key on input file.");
    }
    beam.energy.charge = std::atoi(v.c_str());
    if (!need(in, "ssd", v)) {
        return fail(OMC_E_ARG, "Can not find 'ssd' key on input file.");
    }
    beam.ssd = std::atof(v.c_str());
    if (beam.ssd < 0) {
        return fail(OMC_E_ARG, "SSD must be greater than zero.");
    }
    long ncase = 0;
    int nbatch = 0;
    if (!need(in, "ncase", v)) return fail(OMC_E_ARG, "Can not find 'ncase' key on input file.");
    ncase = std::atol(v.c_str());
    if (!need(in, "nbatch", v)) return fail(OMC_E_ARG, "Can not find 'nbatch' key on input file.");
    nbatch = std::atoi(v.c_str());
    unsigned long long seed = 97ull << 32 | 33ull;
    if (in.get("rng seeds", v)) {
        int a = 0, b = 0;
        if (std::sscanf(v.c_str(), "%d %d", &a, &b) == 2) seed = ((unsigned long long)a << 32) | (unsigned)b;
    }

    omc_phantom P{ph.nx, ph.ny, ph.nz, ph.xb.data(), ph.yb.data(), ph.zb.data(), ph.med.data(), ph.rho.data()};
    omc_engine *eng = nullptr;
    if ((rc = omc_engine_create(tab, &P, &opt, &eng))) {
        return fail(rc, omc_last_error());
    }
    std::vector<double> dose(ph.nvox()), unc(ph.nvox());
    double stats[6] = {0};
    rc = omc_run_beam(eng, &beam, ncase, nbatch, seed, mode, dose.data(), unc.data(), stats);
    if (rc) {
        std::string m = omc_engine_last_error(eng);
        omc_engine_destroy(eng);
        return fail(rc, m);
    }
    if (verbose) {
        std::printf("Total number of particle histories: %.0f\n", stats[0]);
        std::printf("Transport time on the device : %8.4f seconds (%.3e histories/s)\n", stats[1],
                    stats[0] / stats[1]);
        if (stats[4] > 0) std::printf("Fraction of incident energy deposited in the phantom: %5.4f\n", stats[3] / stats[4]);
    }
    rc = write_3ddose(strip_spaces(outdir) + out_name + ".3ddose", ph, dose, unc);
    omc_engine_destroy(eng);
    return rc;
}
