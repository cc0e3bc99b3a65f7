// Physics table builder: PEGS4 reader and the interpolation tables every
// transport kernel reads.  A from-scratch implementation of the maths of
// ompMC's initMediaData chain (src/ompmc.c:5468-5961 and the functions it
// calls); each builder cites the reference lines whose results it must
// reproduce element by element.  Errors are returned, never exit().
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>

#include "omc_host.h"

namespace omc {
namespace {

bool read_all(const std::string &path, std::string &out) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    std::ostringstream ss;
    ss << f.rdbuf();
    out = ss.str();
    return true;
}

std::string trim(const std::string &s) {
    size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

// `KEY=VALUE, KEY=VALUE` line of a PEGS4 header into a lookup.
void parse_kv_line(const std::string &line, std::vector<std::pair<std::string, std::string>> &kv) {
    std::stringstream ss(line);
    std::string tok;
    while (std::getline(ss, tok, ',')) {
        size_t eq = tok.find('=');
        if (eq == std::string::npos) continue;
        kv.emplace_back(strip_spaces(tok.substr(0, eq)), trim(tok.substr(eq + 1)));
    }
}

// ---------------------------------------------------------------- PEGS4
// Reads the requested MEDIUM= blocks (ompmc.c:5507-5961): composition,
// rlc/ae/ap/ue/up, meke, delcm, blcc, xcc, eke0/eke1 and the 16 coefficient
// arrays per electron energy bin; lengths scaled from radiation lengths to cm.
int read_pegs(const std::string &path, const std::vector<std::string> &media,
              std::vector<PegsMedium> &out, std::string &err) {
    std::ifstream f(path);
    if (!f) {
        err = "unable to open pegs file: " + path;
        return -2;
    }
    out.assign(media.size(), PegsMedium());
    std::vector<bool> found(media.size(), false);
    size_t nfound = 0;
    std::string line;
    while (nfound < media.size() && std::getline(f, line)) {
        if (line.rfind(" MEDIUM=", 0) != 0) continue;
        std::string nm = line.substr(8, 24);
        nm = nm.substr(0, nm.find(' '));
        int imed = -1;
        for (size_t i = 0; i < media.size(); i++)
            if (!found[i] && media[i] == nm) { imed = (int)i; break; }
        if (imed < 0) continue;
        PegsMedium &m = out[imed];
        m.name = nm;
        std::getline(f, line);
        std::vector<std::pair<std::string, std::string>> kv;
        parse_kv_line(line, kv);
        for (auto &p : kv) {
            if (p.first == "RHO") m.rho = std::atof(p.second.c_str());
            else if (p.first == "NE") m.ne = std::atoi(p.second.c_str());
        }
        if (m.ne <= 0 || m.ne > MXELEMENT) { err = "bad NE for medium " + nm; return -3; }
        for (int e = 0; e < m.ne; e++) {
            std::getline(f, line);
            kv.clear();
            parse_kv_line(line, kv);
            Element el;
            for (auto &p : kv) {
                if (p.first == "ASYM") el.symbol = strip_spaces(p.second);
                else if (p.first == "Z") el.z = std::atof(p.second.c_str());
                else if (p.first == "A") el.wa = std::atof(p.second.c_str());
                else if (p.first == "PZ") el.pz = std::atof(p.second.c_str());
                else if (p.first == "RHOZ") el.rhoz = std::atof(p.second.c_str());
            }
            m.elements.push_back(el);
        }
        std::getline(f, line);
        if (std::sscanf(line.c_str(), "%lf %lf %lf %lf %lf", &m.rlc, &m.ae, &m.ap, &m.ue, &m.up) != 5) {
            err = "bad rlc/ae/ap/ue/up line for medium " + nm;
            return -3;
        }
        m.te = m.ae - RM;
        m.thmoll = m.te * 2 + RM;
        std::getline(f, line);
        int ints[7];
        if (std::sscanf(line.c_str(), "%d %d %d %d %d %d %d", &ints[0], &ints[1], &ints[2], &ints[3],
                        &ints[4], &ints[5], &ints[6]) != 7) {
            err = "bad array-size line for medium " + nm;
            return -3;
        }
        m.meke = ints[3];
        if (m.meke <= 1 || m.meke > MXEKE) { err = "MEKE out of range for medium " + nm; return -3; }
        // six lines of brems/pair fit coefficients, then a seventh that the
        // reference parses into unused variables (ompmc.c:5873-5880)
        for (int i = 0; i < 7; i++) std::getline(f, line);
        // from here on the block is a whitespace-separated number stream
        double v[14];
        for (double &x : v)
            if (!(f >> x)) { err = "truncated PEGS block for " + nm; return -3; }
        // v: dl6, delcm, alphi1, alphi2, bpar1, bpar2, delpos1, delpos2,
        //    xr0, teff0, blcc, xcc, eke0, eke1
        m.delcm = v[1];
        m.blcc = v[10];
        m.xcc = v[11];
        m.eke0 = v[12];
        m.eke1 = v[13];
        std::vector<double> *arr[16] = {&m.esig0, &m.esig1, &m.psig0, &m.psig1, &m.ededx0, &m.ededx1,
                                        &m.pdedx0, &m.pdedx1, &m.ebr10, &m.ebr11, &m.pbr10, &m.pbr11,
                                        &m.pbr20, &m.pbr21, &m.tmxs0, &m.tmxs1};
        for (auto *a : arr) a->assign(m.meke, 0.0);
        for (int k = 0; k < m.meke; k++)
            for (auto *a : arr)
                if (!(f >> (*a)[k])) { err = "truncated PEGS arrays for " + nm; return -3; }
        std::getline(f, line);
        // lengths in radiation lengths -> cm (ompmc.c:5915-5928)
        double dfacti = 1.0 / m.rlc;
        m.blcc *= dfacti;
        for (int k = 0; k < m.meke; k++) {
            m.esig0[k] *= dfacti; m.psig0[k] *= dfacti; m.ededx0[k] *= dfacti; m.pdedx0[k] *= dfacti;
            m.pdedx1[k] *= dfacti; m.esig1[k] *= dfacti; m.psig1[k] *= dfacti; m.ededx1[k] *= dfacti;
        }
        m.xcc *= std::sqrt(dfacti);
        found[imed] = true;
        nfound++;
    }
    if (nfound < media.size()) {
        err = "media not found in pegs file:";
        for (size_t i = 0; i < media.size(); i++)
            if (!found[i]) err += " " + media[i];
        return -4;
    }
    return 0;
}

// ---------------------------------------------------------- photon tables
// XCOM element data: per element, n then n pairs (ln E, ln sigma)
// (ompmc.c:217-279).  Only the first MXELEMENT elements are used.
struct Xcom {
    std::vector<std::vector<double>> le, ls;
};

int read_xcom(const std::string &path, Xcom &x, std::string &err) {
    std::ifstream f(path);
    if (!f) { err = "unable to open cross-section file: " + path; return -2; }
    x.le.resize(MXELEMENT);
    x.ls.resize(MXELEMENT);
    for (int z = 0; z < MXELEMENT; z++) {
        int n;
        if (!(f >> n) || n <= 0) { err = "bad cross-section file: " + path; return -3; }
        x.le[z].resize(n);
        x.ls[z].resize(n);
        for (int j = 0; j < n; j++)
            if (!(f >> x.le[z][j] >> x.ls[z][j])) { err = "truncated cross-section file: " + path; return -3; }
    }
    return 0;
}

// Per-energy-bin cross section of a medium from element data, log-log
// interpolation on the MXGE grid (ompmc.c:324-422).  `thr` > 0 selects the
// threshold treatment for pair (2m) and triplet (4m): the data are divided by
// (1 - thr/E)^3, a point at the threshold is prepended, and the result is
// multiplied back above threshold.
std::vector<double> medium_xsec(const Xcom &x, const std::vector<double> &zs, const std::vector<double> &pzs,
                                double thr, double ge0, double ge1) {
    std::vector<double> res(MXGE, 0.0);
    for (size_t e = 0; e < zs.size(); e++) {
        int z = (int)(zs[e] + 0.5) - 1;
        std::vector<double> le, ls;
        if (thr > 0) {
            le.push_back(std::log(thr));
            ls.push_back(0.0);
            for (size_t j = 0; j < x.le[z].size(); j++) {
                le.push_back(x.le[z][j]);
                ls.push_back(x.ls[z][j] - 3.0 * std::log(1.0 - thr / std::exp(x.le[z][j])));
            }
            ls[0] = ls[1];
        } else {
            le = x.le[z];
            ls = x.ls[z];
        }
        int n = (int)le.size();
        for (int j = 0; j < MXGE; j++) {
            double gle = ((double)(j + 1) - ge0) / ge1;
            double en = std::exp(gle);
            double sig = 0.0;
            if (gle < le[0] || gle >= le[n - 1]) {
                if (thr > 0 && gle >= le[0]) sig = std::exp(ls[n - 1]);
            } else {
                int k = 0;
                while (k < n - 1 && !(gle >= le[k] && gle < le[k + 1])) k++;
                double p = (gle - le[k]) / (le[k + 1] - le[k]);
                sig = std::exp(p * ls[k + 1] + (1.0 - p) * ls[k]);
            }
            if (thr > 0 && en > thr) sig *= (1.0 - thr / en) * (1.0 - thr / en) * (1.0 - thr / en);
            res[j] += pzs[e] * sig;
        }
    }
    return res;
}

// Free-electron Klein-Nishina total cross section per electron (ompmc.c:424-443).
double klein_nishina(double e) {
    const double con = 0.1274783851;
    double ko = e / RM;
    if (ko < 0.01) return 8.0 * con / 3.0 * (1.0 - ko * (2.0 - ko * (5.2 - 13.3 * ko))) / RM;
    double c1 = 1.0 / (ko * ko);
    double c2 = 1.0 - 2.0 * (1.0 + ko) * c1;
    double c3 = (1.0 + 2.0 * ko) * c1;
    double eps2 = 1.0, eps1 = 1.0 / (1.0 + 2.0 * ko);
    return (c1 * (1.0 / eps1 - 1.0 / eps2) + c2 * std::log(eps2 / eps1) + eps2 * (c3 + 0.5 * eps2) -
            eps1 * (c3 + 0.5 * eps1)) / e * con;
}

// Slope/intercept pairs of a piecewise-linear function of ln E sampled at
// the grid points x_j = (j+1 - c0)/c1: interval j-1 joins points j-1 and j;
// the last interval repeats the previous slope (ompmc.c:600-639).
void pwl_fit(const std::vector<double> &val, int n, double c0, double c1, double *a0, double *a1) {
    double xlast = 0;
    for (int j = 1; j < n; j++) {
        double xj = ((double)(j + 1) - c0) / c1;
        a1[j - 1] = (val[j] - val[j - 1]) * c1;
        a0[j - 1] = val[j] - a1[j - 1] * xj;
        xlast = xj;
    }
    a1[n - 1] = a1[n - 2];
    a0[n - 1] = val[n - 1] - a1[n - 1] * xlast;
}

int build_photon(const DataPaths &p, Tables &t, std::string &err) {
    Xcom photo, rayl, pair, trip;
    std::string d = p.data_folder;
    int rc;
    if ((rc = read_xcom(d + "xcom_photo.data", photo, err))) return rc;
    if ((rc = read_xcom(d + "xcom_rayleigh.data", rayl, err))) return rc;
    if ((rc = read_xcom(d + "xcom_pair.data", pair, err))) return rc;
    if ((rc = read_xcom(d + "xcom_triplet.data", trip, err))) return rc;
    int nmed = t.nmed;
    t.ge0.assign(nmed, 0); t.ge1.assign(nmed, 0);
    for (auto *v : {&t.gmfp0, &t.gmfp1, &t.gbr10, &t.gbr11, &t.gbr20, &t.gbr21, &t.cohe0, &t.cohe1})
        v->assign((size_t)nmed * MXGE, 0.0);
    for (int i = 0; i < nmed; i++) {
        const PegsMedium &m = t.pegs[i];
        t.ge1[i] = (double)(MXGE - 1) / std::log(m.up / m.ap);
        t.ge0[i] = 1.0 - t.ge1[i] * std::log(m.ap);
        double sumA = 0, sumZ = 0;
        std::vector<std::pair<double, double>> zp;
        for (auto &el : m.elements) {
            sumA += el.pz * el.wa;
            sumZ += el.pz * el.z;
            zp.emplace_back(el.z, el.pz);
        }
        for (auto &q : zp)
            if ((int)(q.first + 0.5) > MXELEMENT) { err = "element beyond Z=50 in " + m.name; return -5; }
        std::stable_sort(zp.begin(), zp.end(), [](auto &a, auto &b) { return a.first < b.first; });
        std::vector<double> zs, pzs;
        for (auto &q : zp) { zs.push_back(q.first); pzs.push_back(q.second); }
        double con2 = m.rho / (sumA * 1.6605655);
        auto s_ph = medium_xsec(photo, zs, pzs, 0.0, t.ge0[i], t.ge1[i]);
        auto s_ra = medium_xsec(rayl, zs, pzs, 0.0, t.ge0[i], t.ge1[i]);
        auto s_pa = medium_xsec(pair, zs, pzs, 2.0 * RM, t.ge0[i], t.ge1[i]);
        auto s_tr = medium_xsec(trip, zs, pzs, 4.0 * RM, t.ge0[i], t.ge1[i]);
        std::vector<double> gmfp(MXGE), gbr1(MXGE), gbr2(MXGE), cohe(MXGE);
        for (int j = 0; j < MXGE; j++) {
            double gle = ((double)(j + 1) - t.ge0[i]) / t.ge1[i];
            double skn = sumZ * klein_nishina(std::exp(gle));
            double sp = s_pa[j] + s_tr[j];
            double sigma = skn + sp + s_ph[j];
            gmfp[j] = 1.0 / (sigma * con2);
            gbr1[j] = sp / sigma;
            gbr2[j] = gbr1[j] + skn / sigma;
            cohe[j] = sigma / (s_ra[j] + sigma);
        }
        size_t o = (size_t)i * MXGE;
        pwl_fit(gmfp, MXGE, t.ge0[i], t.ge1[i], &t.gmfp0[o], &t.gmfp1[o]);
        pwl_fit(gbr1, MXGE, t.ge0[i], t.ge1[i], &t.gbr10[o], &t.gbr11[o]);
        pwl_fit(gbr2, MXGE, t.ge0[i], t.ge1[i], &t.gbr20[o], &t.gbr21[o]);
        pwl_fit(cohe, MXGE, t.ge0[i], t.ge1[i], &t.cohe0[o], &t.cohe1[o]);
    }
    return 0;
}

// -------------------------------------------------------------- Rayleigh
// Form-factor CDF tables and pmax(E) (ompmc.c:821-1025; EGSnrc
// prepare_rayleigh_data).  The integral of F^2 x dx^2 between grid points
// uses the local power law F ~ x^b.
int build_rayleigh(const DataPaths &p, Tables &t, std::string &err) {
    std::ifstream f(p.pgs4form_file);
    if (!f) { err = "unable to open pgs4form file: " + p.pgs4form_file; return -2; }
    std::vector<double> xval(MXRAYFF);
    std::vector<std::vector<double>> aff(MXELEMENT, std::vector<double>(MXRAYFF));
    for (auto &v : xval)
        if (!(f >> v)) { err = "bad pgs4form file"; return -3; }
    for (auto &row : aff)
        for (auto &v : row)
            if (!(f >> v)) { err = "bad pgs4form file"; return -3; }
    int nmed = t.nmed;
    for (auto *v : {&t.xgrid, &t.fcum, &t.b_array, &t.c_array}) v->assign((size_t)nmed * MXRAYFF, 0.0);
    t.i_array.assign((size_t)nmed * RAYCDFSIZE, 0);
    t.pmax0.assign((size_t)nmed * MXGE, 0.0);
    t.pmax1.assign((size_t)nmed * MXGE, 0.0);
    for (int i = 0; i < nmed; i++) {
        const PegsMedium &m = t.pegs[i];
        double *x = &t.xgrid[(size_t)i * MXRAYFF];
        double *fc = &t.fcum[(size_t)i * MXRAYFF];
        double *ba = &t.b_array[(size_t)i * MXRAYFF];
        double *ca = &t.c_array[(size_t)i * MXRAYFF];
        int *ia = &t.i_array[(size_t)i * RAYCDFSIZE];
        std::vector<double> ff(MXRAYFF), pe(MXGE);
        for (int j = 0; j < MXRAYFF; j++) {
            x[j] = xval[j];
            double s = 0;
            for (auto &el : m.elements) {
                int z = (int)el.z - 1;
                if (z < 0 || z >= MXELEMENT) { err = "element beyond Z=50 in " + m.name; return -5; }
                s += el.pz * std::pow(aff[z][j], 2);
            }
            ff[j] = std::sqrt(s);
        }
        if (x[0] < 1.0E-6) x[0] = 0.0001;
        double emin = std::exp((1.0 - t.ge0[i]) / t.ge1[i]);
        double emax = std::exp((MXGE - t.ge0[i]) / t.ge1[i]);
        // an exactly-zero form factor becomes the smallest subnormal, so the
        // logarithms below stay finite (ompmc.c:869-892)
        for (auto &v : ff)
            if (v == 0.0 && !std::signbit(v)) v = std::numeric_limits<double>::denorm_min();
        auto seg = [&](double f2, double x1, double x2, double b) {
            double p1 = std::pow(x1, 2.0 * b);
            return f2 * (std::pow(x2, 2) * std::pow(x2, 2.0 * b) - std::pow(x1, 2) * p1) / ((1.0 + b) * p1);
        };
        double sum0 = 0.0;
        fc[0] = 0.0;
        for (int j = 0; j < MXRAYFF - 1; j++) {
            double b = std::log(ff[j + 1] / ff[j]) / std::log(x[j + 1] / x[j]);
            ba[j] = b;
            sum0 += seg(std::pow(ff[j], 2), x[j], x[j + 1], b);
            fc[j + 1] = sum0;
        }
        // the last b is never defined by the reference; it is never read
        ba[MXRAYFF - 1] = 0.0;
        double dle = std::log(emax / emin) / ((double)MXGE - 1.0);
        int idx = 1;
        for (int j = 1; j <= MXGE; j++) {
            double e = emin * std::exp(dle * ((double)j - 1.0));
            double xmax = 20.607544 * 2.0 * e / RM;
            int k = 1;
            while (k <= MXRAYFF - 1 && !(xmax >= x[k - 1] && xmax < x[k])) k++;
            idx = k;
            pe[j - 1] = fc[idx - 1] + seg(std::pow(ff[idx - 1], 2), x[idx - 1], xmax, ba[idx - 1]);
        }
        ia[RAYCDFSIZE - 1] = idx;
        double anorm = 1.0 / std::sqrt(pe[MXGE - 1]);
        double anorm1 = 1.005 / pe[MXGE - 1];
        double anorm2 = 1.0 / pe[MXGE - 1];
        for (auto &v : pe) {
            v *= anorm1;
            if (v > 1.0) v = 1.0;
        }
        for (int j = 0; j < MXRAYFF; j++) {
            ff[j] *= anorm;
            fc[j] *= anorm2;
            ca[j] = (1.0 + ba[j]) / std::pow(x[j] * ff[j], 2);
        }
        // equiprobable cumulative bins -> first grid interval of each
        double dw = 1.0 / ((double)RAYCDFSIZE - 1.0);
        double xold = x[0];
        int ibin = 1;
        double b = ba[0];
        double px1 = std::pow(x[0], 2.0 * b);
        ia[0] = 1;
        for (int j = 2; j <= RAYCDFSIZE - 1; j++) {
            double w = dw;
            for (;;) {
                double x1 = xold, x2 = x[ibin];
                double tt = std::pow(x1, 2) * std::pow(x1, 2.0 * b);
                double f2 = std::pow(ff[ibin - 1], 2);
                double aux = f2 * (std::pow(x2, 2) * std::pow(x2, 2.0 * b) - tt) / ((1.0 + b) * px1);
                if (aux > w) {
                    xold = std::exp(std::log(tt + w * (1.0 + b) * px1 / f2) / (2.0 + 2.0 * b));
                    ia[j - 1] = ibin;
                    break;
                }
                w -= aux;
                xold = x2;
                ibin++;
                if (ibin >= MXRAYFF) { err = "Rayleigh CDF construction ran off the grid"; return -6; }
                b = ba[ibin - 1];
                px1 = std::pow(xold, 2.0 * b);
            }
        }
        for (int j = 0; j < MXRAYFF; j++) ba[j] = 0.5 / (1.0 + ba[j]);
        double *p0 = &t.pmax0[(size_t)i * MXGE], *p1 = &t.pmax1[(size_t)i * MXGE];
        for (int j = 0; j < MXGE - 1; j++) {
            double gle = ((j + 1) - t.ge0[i]) / t.ge1[i];
            p1[j] = (pe[j + 1] - pe[j]) * t.ge1[i];
            p0[j] = pe[j] - p1[j] * gle;
        }
        p0[MXGE - 1] = p0[MXGE - 2];
        p1[MXGE - 1] = p1[MXGE - 2];
    }
    return 0;
}

// ------------------------------------------------------- pair / brems
// Screening-rejection coefficients (ompmc.c:1166-1336; EGSnrc fix_brems and
// $INITIALIZE-PAIR-ANGLE).
double coulomb_fc(double z) {
    double a2 = std::pow(FSC * z, 2);
    return a2 * (1.0 / (1.0 + a2) + 0.20206 - 0.0369 * a2 + 0.0083 * a2 * a2 - 0.002 * a2 * a2 * a2);
}

double atomic_xi(double z, double fc) {
    if (z == 4) return 5.924 / (4.710 - fc);
    if (z == 3) return 5.805 / (4.740 - fc);
    if (z == 2) return 5.621 / (4.790 - fc);
    if (z == 1) return 6.144 / (5.310 - fc);
    return std::log(1194.0 * std::pow(z, -2.0 / 3.0)) / std::log(184.15 * std::pow(z, -1.0 / 3.0)) - fc;
}

void build_pair(Tables &t) {
    int nmed = t.nmed;
    for (auto *v : {&t.dl1, &t.dl2, &t.dl3, &t.dl4, &t.dl5, &t.dl6}) v->assign((size_t)nmed * 8, 0.0);
    for (auto *v : {&t.bpar0, &t.bpar1, &t.delcm, &t.zbrang}) v->assign(nmed, 0.0);
    for (int im = 0; im < nmed; im++) {
        const PegsMedium &m = t.pegs[im];
        double zt = 0, zb = 0, zf = 0;
        for (auto &el : m.elements) {
            double fc = coulomb_fc(el.z);
            double xi = atomic_xi(el.z, fc);
            double aux = el.pz * el.z * (el.z + xi);
            zt += aux;
            zb -= aux * std::log(el.z) / 3.0;
            zf += aux * fc;
        }
        double zv = (zb - zf) / zt, zg = zb / zt;
        double fmax1 = 2.0 * (20.863 + 4.0 * zg) - 2.0 * (20.029 + 4.0 * zg) / 3.0;
        double fmax2 = 2.0 * (20.863 + 4.0 * zv) - 2.0 * (20.029 + 4.0 * zv) / 3.0;
        double *d1 = &t.dl1[im * 8], *d2 = &t.dl2[im * 8], *d3 = &t.dl3[im * 8];
        double *d4 = &t.dl4[im * 8], *d5 = &t.dl5[im * 8], *d6 = &t.dl6[im * 8];
        // brems: screening functions phi1 (rows 0, 2) and phi2 (rows 1, 3),
        // without (zg) and with (zv) the Coulomb correction
        const double zz[2] = {zg, zv};
        const double fm[2] = {fmax1, fmax2};
        for (int c = 0; c < 2; c++) {
            int r = 2 * c;
            d1[r] = (20.863 + 4.0 * zz[c]) / fm[c]; d2[r] = -3.242 / fm[c]; d3[r] = 0.625 / fm[c];
            d4[r] = (21.12 + 4.0 * zz[c]) / fm[c]; d5[r] = -4.184 / fm[c]; d6[r] = 0.952;
            d1[r + 1] = (20.029 + 4.0 * zz[c]) / fm[c]; d2[r + 1] = -1.93 / fm[c]; d3[r + 1] = -0.086 / fm[c];
            d4[r + 1] = (21.12 + 4.0 * zz[c]) / fm[c]; d5[r + 1] = -4.184 / fm[c]; d6[r + 1] = 0.952;
        }
        // pair: 3*phi1 - phi2 (rows 4, 6) and 3*phi1 + phi2 (rows 5, 7)
        for (int c = 0; c < 2; c++) {
            int r = 4 + 2 * c;
            double z = zz[c];
            d1[r] = 3.0 * (20.863 + 4.0 * z) - (20.029 + 4.0 * z);
            d2[r] = 3.0 * (-3.242) - (-1.930);
            d3[r] = 3.0 * 0.625 - (-0.086);
            d4[r] = 2.0 * 21.12 + 8.0 * z;
            d5[r] = 2.0 * (-4.184);
            d6[r] = 0.952;
            d1[r + 1] = 3.0 * (20.863 + 4.0 * z) + (20.029 + 4.0 * z);
            d2[r + 1] = 3.0 * (-3.242) + (-1.930);
            d3[r + 1] = 3.0 * 0.625 + (-0.086);
            d4[r + 1] = 4.0 * 21.12 + 16.0 * z;
            d5[r + 1] = 4.0 * (-4.184);
            d6[r + 1] = 0.952;
        }
        t.bpar1[im] = d1[6] / (3.0 * d1[7] + d1[6]);
        t.bpar0[im] = 12.0 * d1[7] / (3.0 * d1[7] + d1[6]);
        double zbr = 0, pzn = 0;
        for (auto &el : m.elements) {
            zbr += el.pz * el.z * (el.z + 1.0);
            pzn += el.pz;
        }
        t.zbrang[im] = 8.116224E-05 * std::pow(zbr / pzn, 1.0 / 3.0);
        t.delcm[im] = m.delcm;
    }
}

// ------------------------------------------------------- MS surface
// msnew.data: per (lambda, q) block 32 u, 32 f, 31 w, 31 i; f becomes the
// relative slope f[k+1]/f[k]-1 and i a 0-based alias (ompmc.c:3219-3298).
int read_msnew(const DataPaths &p, Tables &t, std::string &err) {
    std::ifstream f(p.data_folder + "msnew.data");
    if (!f) { err = "unable to open " + p.data_folder + "msnew.data"; return -2; }
    t.ums.assign(NMS, 0.0); t.fms.assign(NMS, 0.0); t.wms.assign(NMS, 0.0); t.ims.assign(NMS, 0);
    for (int i = 0; i <= MXL_MS; i++)
        for (int j = 0; j <= MXQ_MS; j++) {
            int o = (i * (MXQ_MS + 1) + j) * (MXU_MS + 1);
            bool ok = true;
            for (int k = 0; k <= MXU_MS; k++) ok = ok && (f >> t.ums[o + k]);
            for (int k = 0; k <= MXU_MS; k++) ok = ok && (f >> t.fms[o + k]);
            for (int k = 0; k < MXU_MS; k++) ok = ok && (f >> t.wms[o + k]);
            for (int k = 0; k < MXU_MS; k++) ok = ok && (f >> t.ims[o + k]);
            if (!ok) { err = "truncated msnew.data"; return -3; }
            for (int k = 0; k < MXU_MS; k++) {
                t.fms[o + k] = t.fms[o + k + 1] / t.fms[o + k] - 1.0;
                t.ims[o + k] -= 1;
            }
            t.fms[o + MXU_MS] = t.fms[o + MXU_MS - 1];
        }
    t.dllambi = 1.0 / ((std::log(LAMBMAX_MS) - std::log(LAMBMIN_MS)) / MXL_MS);
    t.dqmsi = 1.0 / (QMAX_MS / MXQ_MS);
    return 0;
}

// -------------------------------------------------------------- spin
// Spin rejection surface and the PWA corrections to the screening parameter
// and to the first and second MS moments (ompmc.c:2394-2965).  The file
// header is float32; the energy-grid arithmetic is kept in float where the
// reference does it in float, so the grid matches bit for bit.
int build_spin(const DataPaths &p, Tables &t, std::string &err) {
    std::string buf;
    if (!read_all(p.data_folder + "spinms.data", buf)) {
        err = "unable to open " + p.data_folder + "spinms.data";
        return -2;
    }
    if (buf.size() < 1104) { err = "spinms.data too short"; return -3; }
    const float *fb = reinterpret_cast<const float *>(buf.data());
    const uint16_t *sb = reinterpret_cast<const uint16_t *>(buf.data());
    float espin_min = fb[9], espin_max = fb[10], b2spin_min = fb[11], b2spin_max = fb[12];
    t.b2spin_min = (double)b2spin_min;
    const int nener = MXE_SPIN;
    double earray[MXE_SPIN1 + 2];
    {
        double dloge = std::log((double)(espin_max / espin_min)) / (double)nener;
        double eloge = std::log((double)espin_min);
        earray[0] = espin_min;
        for (int i = 1; i <= nener; i++) {
            eloge += dloge;
            earray[i] = std::exp(eloge);
        }
        double dbeta2 = (float)((b2spin_max - b2spin_min) / nener);
        double beta2 = b2spin_min;
        earray[nener + 1] = espin_max;
        for (int i = nener + 2; i <= 2 * nener + 1; i++) {
            beta2 += dbeta2;
            earray[i] = beta2 < 0.999 ? RM * 1000.0 * (1.0 / std::sqrt(1.0 - beta2) - 1) : 50585.1;
        }
    }
    espin_min = (float)(espin_min / 1000.0);
    espin_max = (float)(espin_max / 1000.0);
    t.dleneri = 1.0 / (std::log((double)(espin_max / espin_min)) / MXE_SPIN);
    t.espml = std::log((double)espin_min);
    t.dbeta2i = 1.0 / (double)(float)((b2spin_max - b2spin_min) / MXE_SPIN);
    t.dqq1i = 1.0 / (0.5 / MXQ_SPIN);

    int nmed = t.nmed;
    const int NE1 = MXE_SPIN1 + 1;
    const int NSURF = (MXQ_SPIN + 1) * (MXU_SPIN + 1);
    t.spin_rej.assign((size_t)nmed * NSPIN_PER_MED, 0.0);
    for (auto *v : {&t.etae_ms0, &t.etae_ms1, &t.etap_ms0, &t.etap_ms1, &t.q1ce_ms0, &t.q1ce_ms1, &t.q1cp_ms0,
                    &t.q1cp_ms1, &t.q2ce_ms0, &t.q2ce_ms1, &t.q2cp_ms0, &t.q2cp_ms1, &t.blcce0, &t.blcce1})
        v->assign((size_t)nmed * MXEKE, 0.0);
    const double tf2 = (137.03604 * 0.88534138) * (137.03604 * 0.88534138);
    size_t nrec_avail = buf.size() / 1104;

    for (int im = 0; im < nmed; im++) {
        const PegsMedium &m = t.pegs[im];
        double eta_a[2][NE1] = {}, c_a[2][NE1] = {}, g_a[2][NE1] = {};
        double sum_z2 = 0, sum_z = 0;
        double *sr = &t.spin_rej[(size_t)im * NSPIN_PER_MED];
        for (auto &el : m.elements) {
            double z = el.z;
            int iz = (int)(z + 0.5);
            double tmp = z * (z + 1.0) * el.pz;
            sum_z2 += tmp;
            sum_z += el.pz * z;
            double z23 = std::pow(z, 2.0 / 3.0);
            for (int iq = 0; iq < 2; iq++)
                for (int i = 0; i < NE1; i++) {
                    size_t rec = 1 + (size_t)(iz - 1) * 4 * (nener + 1) + 2 * iq * (nener + 1) + i;
                    if (rec >= nrec_avail) { err = "spinms.data lacks element Z=" + std::to_string(iz); return -3; }
                    const float *r = fb + 276 * rec;
                    double dum1 = r[0], dum2 = r[1], dum3 = r[2], aux_o = r[3];
                    eta_a[iq][i] += tmp * std::log(z23 * aux_o);
                    double tau = earray[i] / (1000.0 * RM);
                    double eta = z23 / tf2 * aux_o / 4 / tau / (tau + 2);
                    c_a[iq][i] += tmp * (std::log(1.0 + 1.0 / eta) - 1.0 / (1.0 + eta)) * dum1 * dum3;
                    g_a[iq][i] += tmp * dum2;
                    const uint16_t *s = sb + 552 * rec + 40;
                    double *dst = sr + ((size_t)iq * NE1 + i) * NSURF;
                    for (int j = 0; j <= MXQ_SPIN; j++) {
                        double fmx = r[4 + j];
                        for (int k = 0; k <= MXU_SPIN; k++)
                            dst[j * (MXU_SPIN + 1) + k] += tmp * ((double)s[j * (MXU_SPIN + 1) + k] * fmx / 65535);
                    }
                }
        }
        // scale each rejection row to a maximum of one
        for (int row = 0; row < 2 * NE1 * (MXQ_SPIN + 1); row++) {
            double *r = sr + (size_t)row * (MXU_SPIN + 1);
            double mx = 0.0;
            for (int k = 0; k <= MXU_SPIN; k++) mx = std::max(mx, r[k]);
            for (int k = 0; k <= MXU_SPIN; k++) r[k] /= mx;
        }
        for (int i = 0; i < NE1; i++) {
            double tau = (earray[i] / RM) * 0.001;
            for (int iq = 0; iq < 2; iq++) {
                double aux_o = std::exp(eta_a[iq][i] / sum_z2) / tf2;
                eta_a[iq][i] = 0.26112447 * aux_o * t.blcc[im] / t.xcc[im];
                double eta = aux_o / 4.0 / tau / (tau + 2);
                double l = std::log(1.0 + 1.0 / eta);
                double gam = 3.0 * (1.0 + eta) * (l * (1.0 + 2.0 * eta) - 2.0) / (l * (1.0 + eta) - 1.0);
                g_a[iq][i] = g_a[iq][i] / sum_z2 / gam;
                c_a[iq][i] = c_a[iq][i] / sum_z2 / (l - 1.0 / (1.0 + eta));
            }
        }
        int neke = m.meke;
        double eke0 = t.eke0[im], eke1 = t.eke1[im];
        // screening-parameter correction eta(E) on the electron grid; the
        // index above the last beta^2 node is clamped (the reference reads one
        // element past its row there)
        auto eta_at = [&](int iq, double eil) {
            double e = std::exp(eil);
            if (e <= espin_min) return eta_a[iq][0];
            double aae;
            int je;
            if (e <= espin_max) {
                aae = (eil - t.espml) * t.dleneri;
                je = (int)aae;
                aae -= je;
            } else {
                double tau = e / RM;
                double beta2 = tau * (tau + 2.0) / ((tau + 1.0) * (tau + 1.0));
                aae = (beta2 - t.b2spin_min) * t.dbeta2i;
                je = (int)aae;
                aae -= je;
                je += MXE_SPIN + 1;
            }
            int je1 = std::min(je + 1, MXE_SPIN1);
            if (iq == 0 && je + 1 == MXE_SPIN1 + 1) return (1.0 - aae) * eta_a[0][je] + aae * eta_a[1][0];
            return (1.0 - aae) * eta_a[iq][je] + aae * eta_a[iq][je1];
        };
        auto tab_from = [&](auto fn, std::vector<double> &v0, std::vector<double> &v1, bool copy_ms1_into_ms0) {
            size_t o = (size_t)im * MXEKE;
            double eil = (1.0 - eke0) / eke1;
            double s1 = fn(eil);
            for (int i = 1; i < neke; i++) {
                eil = (i + 1.0 - eke0) / eke1;
                double s2 = fn(eil);
                v1[o + i - 1] = (s2 - s1) * eke1;
                v0[o + i - 1] = s2 - v1[o + i - 1] * eil;
                s1 = s2;
            }
            v1[o + neke - 1] = v1[o + neke - 2];
            v0[o + neke - 1] = copy_ms1_into_ms0 ? v1[o + neke - 2] : v0[o + neke - 2];
        };
        tab_from([&](double eil) { return eta_at(0, eil); }, t.etae_ms0, t.etae_ms1, false);
        tab_from([&](double eil) { return eta_at(1, eil); }, t.etap_ms0, t.etap_ms1, false);

        // first/second moment corrections: natural splines in ln E over the
        // 31 distinct grid energies plus a node of value 1 at max(1e5, ue)
        std::vector<double> el(NE1), fa(NE1);
        for (int i = 0; i <= MXE_SPIN; i++) el[i] = std::log(earray[i] / 1000.0);
        for (int i = MXE_SPIN + 1; i <= MXE_SPIN1 - 1; i++) el[i] = std::log(earray[i + 1] / 1000.0);
        el[NE1 - 1] = m.ue > 1.0E5 ? std::log(m.ue) : std::log(1.0E5);
        auto moment_table = [&](const double (*src)[NE1], int iq, std::vector<double> &v0, std::vector<double> &v1,
                                bool quirk) {
            for (int i = 0; i <= MXE_SPIN; i++) fa[i] = src[iq][i];
            for (int i = MXE_SPIN + 1; i <= MXE_SPIN1 - 1; i++) fa[i] = src[iq][i + 1];
            fa[NE1 - 1] = 1.0;
            Spline sp;
            sp.fit(el, fa);
            tab_from([&](double eil) { return sp(eil); }, v0, v1, quirk);
        };
        // the electron first-moment table ends with its slope copied into the
        // last intercept, as in the reference (ompmc.c:2802-2803)
        moment_table(c_a, 0, t.q1ce_ms0, t.q1ce_ms1, true);
        moment_table(c_a, 1, t.q1cp_ms0, t.q1cp_ms1, false);
        moment_table(g_a, 0, t.q2ce_ms0, t.q2ce_ms1, false);
        moment_table(g_a, 1, t.q2cp_ms0, t.q2cp_ms1, false);

        // remove the scattering power already in discrete Moller events
        // (ompmc.c:2893-2946)
        double tauc = m.te / RM;
        size_t o = (size_t)im * MXEKE;
        auto blcce_at = [&](double eil) {
            double e = std::exp(eil);
            int leil = (int)std::lround(eil * eke1 + eke0) - 1;
            double tau = e / RM;
            if (!(tau > 2.0 * tauc)) return 1.0;
            double sig = t.esig1[o + leil] * eil + t.esig0[o + leil];
            double dedx = t.ededx1[o + leil] * eil + t.ededx0[o + leil];
            sig /= dedx;
            if (!(sig > 1.0E-6)) return 1.0;
            double etap = t.etae_ms1[o + leil] * eil + t.etae_ms0[o + leil];
            double eta = 0.25 * etap * t.xcc[im] / t.blcc[im] / tau / (tau + 2);
            double g_r = (1.0 + 2.0 * eta) * std::log(1.0 + 1.0 / eta) - 2.0;
            double r = (tau + 2.0) / (tau + 1.0);
            double g_m = std::log(0.5 * tau / tauc) + (1.0 + r * r) * std::log(2.0 * (tau - tauc + 2.0) / (tau + 4.0)) -
                         0.25 * (tau + 2.0) * (tau + 2.0 + 2.0 * (2.0 * tau + 1.0) / ((tau + 1.0) * (tau + 1.0))) *
                             std::log((tau + 4.0) * (tau - tauc) / tau / (tau - tauc + 2.0)) +
                         0.5 * (tau - 2.0 * tauc) * (tau + 2.0) * (1.0 / (tau - tauc) - 1.0 / ((tau + 1.0) * (tau + 1.0)));
            g_m = g_m < g_r ? g_m / g_r : 1.0;
            return 1.0 - g_m * sum_z / sum_z2;
        };
        {
            double s1 = 1.0;
            for (int i = 1; i < neke; i++) {
                double eil = ((double)(i + 1) - eke0) / eke1;
                double s2 = blcce_at(eil);
                t.blcce1[o + i - 1] = (s2 - s1) * eke1;
                t.blcce0[o + i - 1] = s2 - t.blcce1[o + i - 1] * eil;
                s1 = s2;
            }
            t.blcce1[o + neke - 1] = t.blcce1[o + neke - 2];
            t.blcce0[o + neke - 1] = t.blcce0[o + neke - 2];
        }
    }
    return 0;
}

// ------------------------------------------- electron range / step tables
// sig/dE maxima and monotonicity, CSDA range table and the maximum CH step
// tmxs (ompmc.c:3338-3529).
void build_electron_ranges(Tables &t) {
    int nmed = t.nmed;
    t.sig_ismonotone.assign(2 * nmed, 1);
    t.esig_e.assign(nmed, 0); t.psig_e.assign(nmed, 0); t.expeke1.assign(nmed, 0);
    t.e_array.assign((size_t)nmed * MXEKE, 0.0);
    t.range_ep.assign((size_t)2 * nmed * MXEKE, 0.0);
    for (int im = 0; im < nmed; im++) {
        size_t o = (size_t)im * MXEKE;
        int neke = t.pegs[im].meke;
        double eke0 = t.eke0[im], eke1 = t.eke1[im];
        double sge = 1.0E-15, sgp = 1.0E-15, olde = -1.0, oldp = -1.0;
        int mone = 1, monp = 1;
        for (int i = 1; i <= neke; i++) {
            double eil = std::log(std::exp(((double)i - eke0) / eke1));
            size_t l = o + i - 1;
            double se = (t.esig1[l] * eil + t.esig0[l]) / (t.ededx1[l] * eil + t.ededx0[l]);
            double sp = (t.psig1[l] * eil + t.psig0[l]) / (t.pdedx1[l] * eil + t.pdedx0[l]);
            sge = std::max(sge, se);
            sgp = std::max(sgp, sp);
            if (se < olde) mone = 0;
            if (sp < oldp) monp = 0;
            olde = se;
            oldp = sp;
        }
        t.sig_ismonotone[im] = mone;
        t.sig_ismonotone[nmed + im] = monp;
        t.esig_e[im] = sge;
        t.psig_e[im] = sgp;

        double *re = &t.range_ep[o], *rp = &t.range_ep[(size_t)nmed * MXEKE + o];
        double ei = std::exp((1.0 - eke0) / eke1);
        t.e_array[o] = ei;
        t.expeke1[im] = std::exp(1.0 / eke1) - 1.0;
        for (int i = 1; i < neke; i++) {
            double eip1 = std::exp(((double)(i + 1) - eke0) / eke1);
            t.e_array[o + i] = eip1;
            // range over one interval: log-linear stopping power and a power
            // series of the resulting exponential integral
            double eke = 0.5 * (eip1 + ei);
            double elke = std::log(eke);
            int lelke = (int)(eke1 * elke + eke0) - 1;
            double r2 = std::pow((eip1 - ei) / eke, 2.0);
            double dp = t.pdedx1[o + lelke] * elke + t.pdedx0[o + lelke];
            double ap = t.pdedx1[o + i - 1] / dp;
            rp[i] = rp[i - 1] + (eip1 - ei) / dp * (1.0 + ap * (1.0 + 2.0 * ap) * r2 / 24.0);
            double de = t.ededx1[o + lelke] * elke + t.ededx0[o + lelke];
            double ae = t.ededx1[o + i - 1] / de;
            re[i] = re[i - 1] + (eip1 - ei) / de * (1.0 + ae * (1.0 + 2.0 * ae) * r2 / 24.0);
            ei = eip1;
        }

        // maximum CH step: the path over which the electron loses the
        // fraction estepx = min(XIMAX * (step of one MS moment), ESTEPE) of
        // its energy; the first point evaluates stopping power in interval 1
        // as the reference does (ompmc.c:3443-3447)
        auto estep = [&](double e, double dedx) {
            double p2 = e * (e + 2.0 * RM);
            double beta2 = p2 / (p2 + RM * RM);
            double chi = t.xcc[im] / (4.0 * p2 * t.blcc[im]);
            double x = 2.0 * p2 * beta2 * dedx / e / t.xcc[im] / (std::log(1.0 + 1.0 / chi) * (1.0 + chi) - 1.0);
            return std::min(x * XIMAX, ESTEPE);
        };
        double eil = (1.0 - eke0) / eke1;
        double e0 = std::exp(eil);
        double dedx0 = t.ededx1[o + 1] * eil + t.ededx0[o + 1];
        double si = estep(e0, dedx0) * e0 / dedx0;
        for (int i = 1; i < neke; i++) {
            double elke = ((double)(i + 1) - eke0) / eke1;
            double eke = std::exp(elke);
            double dedx = t.ededx1[o + i] * elke + t.ededx0[o + i];
            double ekef = (1.0 - estep(eke, dedx)) * eke;
            double sip1;
            int lelkef;
            if (ekef <= t.e_array[o]) {
                sip1 = (t.e_array[o] - ekef) / dedx0;
                lelkef = 0;
            } else {
                double elkef = std::log(ekef);
                lelkef = (int)(eke1 * elkef + eke0 - 1);
                int leip1l = lelkef + 1;
                double eip1l = ((double)(leip1l + 1) - eke0) / eke1;
                double eip1 = t.e_array[o + leip1l];
                double aux = (eip1 - ekef) / eip1;
                double elktmp = 0.5 * (elkef + eip1l + 0.25 * aux * aux * (1.0 + aux * (1.0 + 0.875 * aux)));
                double ektmp = 0.5 * (ekef + eip1);
                double d = t.ededx1[o + lelkef] * elktmp + t.ededx0[o + lelkef];
                double a = t.ededx1[o + lelkef] / d;
                sip1 = (eip1 - ekef) / d * (1.0 + a * (1.0 + 2.0 * a) * (std::pow((eip1 - ekef) / ektmp, 2.0) / 24.0));
            }
            sip1 += re[i] - re[lelkef + 1];
            t.tmxs1[o + i - 1] = (sip1 - si) * eke1;
            t.tmxs0[o + i - 1] = sip1 - t.tmxs1[o + i - 1] * elke;
            si = sip1;
        }
        t.tmxs0[o + neke - 1] = t.tmxs0[o + neke - 2];
        t.tmxs1[o + neke - 1] = t.tmxs1[o + neke - 2];
    }
}

}  // namespace

// --------------------------------------------------------------- spline
// Natural cubic spline through (xs, fs), with the elimination order of
// EGSnrc's set_spline as ompMC has it (ompmc.c:3034-3076), so that the
// tables built on it (the spin moment corrections) agree bit for bit:
// forward pass over the slope differences, back substitution, then the
// polynomial coefficients of each interval.
void Spline::fit(const std::vector<double> &xs, const std::vector<double> &fs) {
    const int n = (int)xs.size();
    x = xs;
    a.assign(n, 0); b.assign(n, 0); c.assign(n, 0); d.assign(n, 0);
    // interval widths, and the change of slope at each inner node
    double prev_slope = 0.0;
    for (int k = 0; k < n - 1; k++) {
        d[k] = xs[k + 1] - xs[k];
        const double slope = (fs[k + 1] - fs[k]) / d[k];
        c[k] = slope - prev_slope;
        prev_slope = slope;
    }
    c[0] = 0.0;
    c[n - 1] = 0.0;
    // forward elimination of the tridiagonal system (diagonal into b)
    double ratio = 0.0, width = 0.0;
    for (int k = 1; k < n - 1; k++) {
        c[k] = c[k] + ratio * c[k - 1];
        b[k] = 2.0 * (xs[k - 1] - xs[k + 1]) - ratio * width;
        width = d[k];
        ratio = width / b[k];
    }
    // back substitution, from the last inner node down
    for (int k = n - 2; k >= 1; k--) c[k] = (d[k] * c[k + 1] - c[k]) / b[k];
    // coefficients of a + q (b + q (c + q d)) on each interval
    for (int k = 0; k < n - 1; k++) {
        const double h = d[k];
        const double dc = c[k + 1] - c[k];
        d[k] = dc / h;
        c[k] = 3.0 * c[k];
        b[k] = (fs[k + 1] - fs[k]) / h - (c[k] + dc) * h;
        a[k] = fs[k];
    }
}

double Spline::operator()(double s) const {
    int n = (int)x.size();
    int idx;
    if (s >= x[n - 1]) idx = n - 2;
    else if (s <= x[0]) idx = 0;
    else idx = (int)(std::upper_bound(x.begin(), x.end(), s) - x.begin()) - 1;
    double q = s - x[idx];
    return a[idx] + q * (b[idx] + q * (c[idx] + q * d[idx]));
}

// ------------------------------------------------------------ driver
int build_tables(const DataPaths &paths, const std::vector<std::string> &media, Tables &t, std::string &err) {
    if (media.empty() || (int)media.size() > MXMED) {
        err = "number of media must be 1.." + std::to_string(MXMED);
        return -1;
    }
    t = Tables();
    t.nmed = (int)media.size();
    t.names = media;
    int rc = read_pegs(paths.pegs_file, media, t.pegs, err);
    if (rc) return rc;
    int nmed = t.nmed;
    // electron tables straight from PEGS
    for (auto *v : {&t.esig0, &t.esig1, &t.psig0, &t.psig1, &t.ededx0, &t.ededx1, &t.pdedx0, &t.pdedx1, &t.ebr10,
                    &t.ebr11, &t.pbr10, &t.pbr11, &t.pbr20, &t.pbr21, &t.tmxs0, &t.tmxs1})
        v->assign((size_t)nmed * MXEKE, 0.0);
    t.eke0.assign(nmed, 0); t.eke1.assign(nmed, 0); t.xcc.assign(nmed, 0); t.blcc.assign(nmed, 0);
    for (int im = 0; im < nmed; im++) {
        const PegsMedium &m = t.pegs[im];
        size_t o = (size_t)im * MXEKE;
        for (int k = 0; k < m.meke; k++) {
            t.esig0[o + k] = m.esig0[k]; t.esig1[o + k] = m.esig1[k];
            t.psig0[o + k] = m.psig0[k]; t.psig1[o + k] = m.psig1[k];
            t.ededx0[o + k] = m.ededx0[k]; t.ededx1[o + k] = m.ededx1[k];
            t.pdedx0[o + k] = m.pdedx0[k]; t.pdedx1[o + k] = m.pdedx1[k];
            t.ebr10[o + k] = m.ebr10[k]; t.ebr11[o + k] = m.ebr11[k];
            t.pbr10[o + k] = m.pbr10[k]; t.pbr11[o + k] = m.pbr11[k];
            t.pbr20[o + k] = m.pbr20[k]; t.pbr21[o + k] = m.pbr21[k];
            t.tmxs0[o + k] = m.tmxs0[k]; t.tmxs1[o + k] = m.tmxs1[k];
        }
        t.eke0[im] = m.eke0;
        t.eke1[im] = m.eke1;
        // Euler's constant absorbed into blcc; xcc squared (ompmc.c:3306-3314)
        t.blcc[im] = 1.16699413758864573 * m.blcc;
        t.xcc[im] = std::pow(m.xcc, 2.0);
    }
    if ((rc = build_photon(paths, t, err))) return rc;
    if ((rc = build_rayleigh(paths, t, err))) return rc;
    build_pair(t);
    if ((rc = read_msnew(paths, t, err))) return rc;
    if ((rc = build_spin(paths, t, err))) return rc;
    build_electron_ranges(t);
    return 0;
}

}  // namespace omc
