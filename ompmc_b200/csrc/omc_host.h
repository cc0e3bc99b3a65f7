// Host-side data model of the dose engine: physics tables, phantom, source
// and run parameters, all built on the host in FP64 and uploaded once.
//
// Array sizes and index conventions follow ompMC so tables compare element by
// element with the reference (ompMC src/ompmc.h:107-435):
//   photon tables   [nmed][MXGE]   indexed by  (int)(ge1*ln E + ge0) - 1
//   electron tables [nmed][MXEKE]  indexed by  (int)(eke1*ln E + eke0) - 1
//   Rayleigh        [nmed][MXRAYFF], spin [nmed][2][32][16][32],
//   MS surface      [64][8][32].
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace omc {

constexpr double RM = 0.5109989461;  // electron rest energy, MeV
constexpr int MXGE = 2000;
constexpr int MXEKE = 500;
constexpr int MXRAYFF = 100;
constexpr int RAYCDFSIZE = 100;
constexpr int MXELEMENT = 50;
constexpr int MXMED = 9;
constexpr int MXE_SPIN = 15;
constexpr int MXE_SPIN1 = 2 * MXE_SPIN + 1;
constexpr int MXQ_SPIN = 15;
constexpr int MXU_SPIN = 31;
constexpr int NSPIN_PER_MED = 2 * (MXE_SPIN1 + 1) * (MXQ_SPIN + 1) * (MXU_SPIN + 1);
constexpr int MXL_MS = 63;
constexpr int MXQ_MS = 7;
constexpr int MXU_MS = 31;
constexpr int NMS = (MXL_MS + 1) * (MXQ_MS + 1) * (MXU_MS + 1);
constexpr double LAMBMIN_MS = 1.0;
constexpr double LAMBMAX_MS = 1.0E5;
constexpr double QMIN_MS = 1.0E-3;
constexpr double QMAX_MS = 0.5;
constexpr double XIMAX = 0.5;
constexpr double ESTEPE = 0.25;
constexpr double EPSEMFP = 1.0E-5;
constexpr double SGMFP = 1.0E-5;
constexpr double SKIN_DEPTH_FOR_BCA = 3.0;
constexpr double HC_INVERSE = 80.65506856998;
constexpr double TWICE_HC2 = 0.000307444456;
constexpr double FSC = 0.00729735255664;

struct Element {
    std::string symbol;
    double z = 0, wa = 0, pz = 0, rhoz = 0;
};

// One PEGS4 medium block (ompMC src/ompmc.c:5507-5961).
struct PegsMedium {
    std::string name;
    double rho = 0;
    int ne = 0;
    std::vector<Element> elements;
    double rlc = 0, ae = 0, ap = 0, ue = 0, up = 0, te = 0, thmoll = 0, delcm = 0;
    int meke = 0;
    double blcc = 0, xcc = 0, eke0 = 0, eke1 = 0;
    // 16 coefficient arrays per energy bin, in file order
    std::vector<double> esig0, esig1, psig0, psig1, ededx0, ededx1, pdedx0, pdedx1;
    std::vector<double> ebr10, ebr11, pbr10, pbr11, pbr20, pbr21, tmxs0, tmxs1;
};

// All tables, laid out as the reference lays them out (FP64).
struct Tables {
    int nmed = 0;
    std::vector<std::string> names;
    std::vector<PegsMedium> pegs;

    // photon, [nmed*MXGE] slope (1) / intercept (0)
    std::vector<double> ge0, ge1, gmfp0, gmfp1, gbr10, gbr11, gbr20, gbr21, cohe0, cohe1;
    // Rayleigh
    std::vector<double> xgrid, fcum, b_array, c_array, pmax0, pmax1;
    std::vector<int> i_array;
    // pair / brems parameters
    std::vector<double> dl1, dl2, dl3, dl4, dl5, dl6, bpar0, bpar1, delcm, zbrang;
    // electron, [nmed*MXEKE]
    std::vector<double> esig0, esig1, psig0, psig1, ededx0, ededx1, pdedx0, pdedx1;
    std::vector<double> ebr10, ebr11, pbr10, pbr11, pbr20, pbr21, tmxs0, tmxs1;
    std::vector<double> blcce0, blcce1, etae_ms0, etae_ms1, etap_ms0, etap_ms1;
    std::vector<double> q1ce_ms0, q1ce_ms1, q1cp_ms0, q1cp_ms1, q2ce_ms0, q2ce_ms1, q2cp_ms0, q2cp_ms1;
    std::vector<double> range_ep;  // [2][nmed][MXEKE]
    std::vector<double> e_array;   // [nmed][MXEKE]
    std::vector<double> eke0, eke1, esig_e, psig_e, xcc, blcc, expeke1;
    std::vector<int> sig_ismonotone;  // [2][nmed]
    // spin
    double b2spin_min = 0, dbeta2i = 0, espml = 0, dleneri = 0, dqq1i = 0;
    std::vector<double> spin_rej;  // [nmed][2][32][16][32]
    // screened Rutherford MS surface
    std::vector<double> ums, fms, wms;
    std::vector<int> ims;
    double dllambi = 0, dqmsi = 0;
};

// Paths of the physics data (the `.inp` keys `pegs file`, `pgs4form file`,
// `data folder`).
struct DataPaths {
    std::string pegs_file, pgs4form_file, data_folder;
};

// Builds every table for the named media.  Returns 0 on success; on failure
// returns a negative status and writes a message to `err`.
int build_tables(const DataPaths &paths, const std::vector<std::string> &media, Tables &t,
                 std::string &err);

// Natural cubic spline through (x[i], f[i]); evaluates like ompMC's
// spline() (ompmc.c:3078-3112): the polynomial of the bracketing interval,
// the first interval below x[0] and the last one above x[n-1].
struct Spline {
    std::vector<double> x, a, b, c, d;
    void fit(const std::vector<double> &xs, const std::vector<double> &fs);
    double operator()(double s) const;
};

// Rectilinear voxel phantom; voxel index v = i + j*nx + k*nx*ny, region
// number ir = v + 1, region 0 is outside (omc_dosxyz.c:124-128, :925-962).
struct Phantom {
    int nx = 0, ny = 0, nz = 0;
    std::vector<double> xb, yb, zb;
    std::vector<int> med;    // 1-based medium index per voxel (0 = vacuum)
    std::vector<double> rho; // density per voxel
    std::vector<std::string> media;
    long nvox() const { return (long)nx * ny * nz; }
};

// Region data per region (size nvox+1) as initRegions sets it.
struct Regions {
    std::vector<int> med;  // -1 = vacuum (region 0 is outside)
    std::vector<double> rhof, pcut, ecut;
};
int build_regions(const Phantom &ph, const Tables &t, double ecut, double pcut, Regions &r,
                  std::string &err);

// Spectrum inverse CDF (omc_dosxyz.c:368-510), INVDIM bins.
struct Spectrum {
    bool mono = true;
    double energy = 0;
    std::vector<double> cdfinv1, cdfinv2;
    double deltak = 1000;
};
int read_spectrum(const std::string &file, Spectrum &s, std::string &err);

// `.inp` key/value store with ompMC's semantics (omc_utilities.c:63-125).
struct Input {
    std::vector<std::pair<std::string, std::string>> items;
    int parse_file(const std::string &path, std::string &err);
    bool get(const char *key, std::string &value) const;
};
std::string strip_spaces(const std::string &s);

int read_egsphant(const std::string &path, Phantom &ph, std::string &err);

}  // namespace omc
