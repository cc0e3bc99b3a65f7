// Host input formats of the dosxyz surface: `.inp` key/value files,
// `.egsphant` phantoms, `.spectrum` files, and the per-region transport data.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

#include "omc_host.h"

namespace omc {

std::string strip_spaces(const std::string &s) {
    std::string o;
    for (char c : s)
        if (!std::isspace((unsigned char)c)) o += c;
    return o;
}

// `key = value` lines; a line containing '#' anywhere is skipped, as are
// blank lines (omc_utilities.c:63-95).  Lookup returns the first item whose
// key CONTAINS the query (strstr semantics, omc_utilities.c:98-119).
int Input::parse_file(const std::string &path, std::string &err) {
    std::ifstream f(path);
    if (!f) {
        err = "unable to open input file: " + path;
        return -2;
    }
    items.clear();
    std::string line;
    while (std::getline(f, line)) {
        if (line.find('#') != std::string::npos) continue;
        bool blank = true;
        for (char c : line)
            if (!std::isspace((unsigned char)c)) { blank = false; break; }
        if (blank) continue;
        size_t eq = line.find('=');
        std::string key = eq == std::string::npos ? line : line.substr(0, eq);
        std::string val = eq == std::string::npos ? "" : line.substr(eq + 1);
        while (!val.empty() && (val.back() == '\r' || val.back() == '\n')) val.pop_back();
        items.emplace_back(key, val);
    }
    return 0;
}

bool Input::get(const char *key, std::string &value) const {
    for (auto &kv : items)
        if (kv.first.find(key) != std::string::npos) {
            value = kv.second;
            return true;
        }
    return false;
}

// `.egsphant`: nmed, names, a dummy line, nx ny nz, boundaries, one digit per
// voxel (rows of x, a blank line per z slice), then densities
// (omc_dosxyz.c:62-152).
int read_egsphant(const std::string &path, Phantom &ph, std::string &err) {
    std::ifstream f(path);
    if (!f) {
        err = "unable to open phantom file: " + path;
        return -2;
    }
    std::string line;
    std::getline(f, line);
    int nmed = std::atoi(line.c_str());
    if (nmed <= 0 || nmed > MXMED) {
        err = "bad number of media in phantom: " + line;
        return -3;
    }
    ph.media.clear();
    for (int i = 0; i < nmed; i++) {
        std::getline(f, line);
        ph.media.push_back(strip_spaces(line));
    }
    std::getline(f, line);
    std::getline(f, line);
    if (std::sscanf(line.c_str(), "%d %d %d", &ph.nx, &ph.ny, &ph.nz) != 3 || ph.nx <= 0 || ph.ny <= 0 || ph.nz <= 0) {
        err = "bad phantom dimensions: " + line;
        return -3;
    }
    ph.xb.resize(ph.nx + 1);
    ph.yb.resize(ph.ny + 1);
    ph.zb.resize(ph.nz + 1);
    for (auto *v : {&ph.xb, &ph.yb, &ph.zb})
        for (auto &x : *v)
            if (!(f >> x)) { err = "truncated phantom boundaries"; return -3; }
    std::getline(f, line);
    long nv = ph.nvox();
    ph.med.assign(nv, 0);
    ph.rho.assign(nv, 0.0);
    for (int k = 0; k < ph.nz; k++) {
        for (int j = 0; j < ph.ny; j++) {
            std::getline(f, line);
            if ((int)line.size() < ph.nx) { err = "truncated phantom media row"; return -3; }
            for (int i = 0; i < ph.nx; i++) {
                int m = line[i] - '0';
                if (m < 0 || m > nmed) { err = "bad medium digit in phantom"; return -3; }
                ph.med[i + (long)j * ph.nx + (long)k * ph.nx * ph.ny] = m;
            }
        }
        std::getline(f, line);
    }
    for (long v = 0; v < nv; v++)
        if (!(f >> ph.rho[v])) { err = "truncated phantom densities"; return -3; }
    return 0;
}

// Per-region medium, density ratio and cut-offs (initRegions,
// omc_dosxyz.c:890-962).  Region 0 is outside (vacuum).  Cut-offs below the
// PEGS thresholds AP/AE are raised to them (the reference leaves the
// electron cut-off unset in that case).
int build_regions(const Phantom &ph, const Tables &t, double ecut, double pcut, Regions &r, std::string &err) {
    long nreg = ph.nvox() + 1;
    r.med.assign(nreg, -1);
    r.rhof.assign(nreg, 0.0);
    r.pcut.assign(nreg, 0.0);
    r.ecut.assign(nreg, 0.0);
    for (long i = 1; i < nreg; i++) {
        int imed = ph.med[i - 1] - 1;
        if (imed >= t.nmed) {
            err = "voxel medium index beyond the media list";
            return -3;
        }
        r.med[i] = imed;
        if (imed < 0) continue;
        const PegsMedium &m = t.pegs[imed];
        r.rhof[i] = ph.rho[i - 1] == 0.0 ? 1.0 : ph.rho[i - 1] / m.rho;
        r.pcut[i] = m.ap <= pcut ? pcut : m.ap;
        r.ecut[i] = m.ae <= ecut ? ecut : m.ae;
    }
    return 0;
}

// `.spectrum`: title; `nbins emin imode`; `E_upper weight` lines; imode 0 is
// counts/bin, 1 counts/MeV.  Builds the INVDIM-point inverse CDF
// (omc_dosxyz.c:368-510).
int read_spectrum(const std::string &file, Spectrum &s, std::string &err) {
    std::ifstream f(file);
    if (!f) {
        err = "unable to open spectrum file: " + file;
        return -2;
    }
    std::string line;
    std::getline(f, line);
    std::getline(f, line);
    int nb = 0, imode = 0;
    double enmin = 0;
    if (std::sscanf(line.c_str(), "%d %lf %d", &nb, &enmin, &imode) != 3 || nb <= 0 || nb > 200) {
        err = "bad spectrum header: " + line;
        return -3;
    }
    std::vector<double> eu(nb), pdf(nb);
    for (int i = 0; i < nb; i++) {
        std::getline(f, line);
        if (std::sscanf(line.c_str(), "%lf %lf", &eu[i], &pdf[i]) != 2) {
            err = "bad spectrum line: " + line;
            return -3;
        }
    }
    if (imode == 1) {
        pdf[0] *= (eu[0] - enmin);
        for (int i = 1; i < nb; i++) pdf[i] *= (eu[i] - eu[i - 1]);
    } else if (imode != 0) {
        err = "invalid spectrum mode";
        return -3;
    }
    std::vector<double> cdf(nb);
    cdf[0] = pdf[0];
    for (int i = 1; i < nb; i++) cdf[i] = cdf[i - 1] + pdf[i];
    double fnorm = 1.0 / cdf[nb - 1];
    for (auto &c : cdf) c *= fnorm;
    const int invdim = 1000;
    s.mono = false;
    s.deltak = invdim;
    double gridsz = 1.0f / s.deltak;
    s.cdfinv1.assign(invdim, 0.0);
    s.cdfinv2.assign(invdim, 0.0);
    for (int k = 0; k < invdim; k++) {
        double ak = (double)k * gridsz;
        int i = 0;
        while (i < nb && !(ak <= cdf[i])) i++;
        if (i >= nb) i = nb - 1;
        s.cdfinv1[k] = i != 0 ? eu[i - 1] : enmin;
        s.cdfinv2[k] = eu[i] - s.cdfinv1[k];
    }
    return 0;
}

}  // namespace omc
