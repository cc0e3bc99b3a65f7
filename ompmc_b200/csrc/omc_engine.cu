// Engine: resident device tables and phantom, batch statistics, and the C
// ABI entry points of include/omcgpu.h.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "omc_engine.h"
#include "omc_event.h"

using namespace omc;

namespace {
std::mutex g_err_mu;
std::string g_err;

int global_err(int code, const std::string &msg) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_err = msg;
    return code;
}
}  // namespace

namespace omc {

// Device allocations the library has made (every one goes through DBuf).
static std::atomic<long long> g_device_allocs{0};

int DBuf::alloc(size_t bytes) {
    release();
    if (bytes == 0) bytes = 16;
    cudaError_t rc = cudaMalloc(&p, bytes);
    if (rc != cudaSuccess) {
        p = nullptr;
        return rc == cudaErrorMemoryAllocation ? OMC_E_NOMEM : OMC_E_CUDA;
    }
    n = bytes;
    g_device_allocs.fetch_add(1, std::memory_order_relaxed);
    return OMC_OK;
}

int set_err(omc_engine *e, int code, const std::string &msg) {
    if (e) e->err = msg;
    global_err(code, msg);
    return code;
}

int cuda_check(omc_engine *e, cudaError_t rc, const char *what) {
    if (rc == cudaSuccess) return OMC_OK;
    return set_err(e, rc == cudaErrorMemoryAllocation ? OMC_E_NOMEM : OMC_E_CUDA,
                   std::string(what) + ": " + cudaGetErrorString(rc));
}

template <typename T>
static int upload(omc_engine *e, DBuf &b, const std::vector<T> &v) {
    int rc = b.alloc(v.size() * sizeof(T));
    if (rc) return set_err(e, rc, "device allocation failed");
    return cuda_check(e, cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
}

template <typename R>
static PL<R> mkpl(double a1, double a0) {
    PL<R> p;
    p.a1 = (R)a1;
    p.a0 = (R)a0;
    return p;
}

// Host tables -> interleaved device layout in precision R (host vectors).
template <typename R>
void make_layout(const Tables &t, const Phantom &ph, const Regions &rg, double ecut, double pcut, int ref_compat,
                 Layout<R> &L) {
    int nmed = t.nmed;
    DevData<R> &d = L.d;
    d = DevData<R>{};
    d.nmed = nmed;
    d.nx = ph.nx;
    d.ny = ph.ny;
    d.nz = ph.nz;
    d.div_nx = FastDiv::make((uint32_t)ph.nx);
    d.div_nxy = FastDiv::make((uint32_t)ph.nx * (uint32_t)ph.ny);
    d.ref_compat = ref_compat;
    d.nsplit = 1;
    // uniform grid and per-medium density maxima (photon delta tracking)
    auto uniform_axis = [](const std::vector<double> &b, double &x0, double &x1, double &inv) {
        int n = (int)b.size() - 1;
        x0 = b[0];
        x1 = b[n];
        double dx = (x1 - x0) / n;
        inv = 1.0 / dx;
        for (int i = 0; i < n; i++)
            if (std::fabs((b[i + 1] - b[i]) - dx) > 1e-6 * dx) return false;
        return dx > 0;
    };
    double ax[3][3];
    bool uni = uniform_axis(ph.xb, ax[0][0], ax[0][1], ax[0][2]);
    uni = uniform_axis(ph.yb, ax[1][0], ax[1][1], ax[1][2]) && uni;
    uni = uniform_axis(ph.zb, ax[2][0], ax[2][1], ax[2][2]) && uni;
    d.uniform = uni ? 1 : 0;
    d.gx0 = (R)ax[0][0]; d.gx1 = (R)ax[0][1]; d.gidx = (R)ax[0][2];
    d.gy0 = (R)ax[1][0]; d.gy1 = (R)ax[1][1]; d.gidy = (R)ax[1][2];
    d.gz0 = (R)ax[2][0]; d.gz1 = (R)ax[2][1]; d.gidz = (R)ax[2][2];
    for (int m = 0; m < D_MXMED; m++) d.rhomax[m] = 0;
    for (size_t r = 1; r < rg.med.size(); r++) {
        int m = rg.med[r];
        if (m >= 0 && m < D_MXMED) d.rhomax[m] = std::max(d.rhomax[m], (R)rg.rhof[r]);
    }
    L.xb.assign(ph.xb.begin(), ph.xb.end());
    L.yb.assign(ph.yb.begin(), ph.yb.end());
    L.zb.assign(ph.zb.begin(), ph.zb.end());
    L.med.assign(rg.med.begin(), rg.med.end());
    L.rhof.assign(rg.rhof.begin(), rg.rhof.end());
    L.ms.assign(nmed, MedS<R>{});
    L.ph.assign((size_t)nmed * D_MXGE, PhBin<R>{});
    L.pmax.assign((size_t)nmed * D_MXGE, PL<R>{});
    L.ray.assign(nmed, Rayl<R>{});
    L.el.assign((size_t)nmed * 2 * D_MXEKE, ElBin<R>{});
    for (int im = 0; im < nmed; im++) {
        const PegsMedium &m = t.pegs[im];
        MedS<R> &s = L.ms[im];
        std::memset(&s, 0, sizeof(s));
        s.ge0 = t.ge0[im]; s.ge1 = t.ge1[im]; s.eke0 = t.eke0[im]; s.eke1 = t.eke1[im];
        s.blcc = t.blcc[im]; s.xcc = t.xcc[im]; s.sige[0] = t.esig_e[im]; s.sige[1] = t.psig_e[im];
        s.te = m.te; s.thmoll = m.thmoll; s.ap = m.ap; s.ae = m.ae;
        s.delcm = t.delcm[im]; s.zbrang = t.zbrang[im]; s.bpar0 = t.bpar0[im]; s.bpar1 = t.bpar1[im];
        s.pcut = m.ap <= pcut ? pcut : m.ap;
        s.ecut = m.ae <= ecut ? ecut : m.ae;
        for (int k = 0; k < 8; k++) {
            s.dl1[k] = t.dl1[im * 8 + k]; s.dl2[k] = t.dl2[im * 8 + k]; s.dl3[k] = t.dl3[im * 8 + k];
            s.dl4[k] = t.dl4[im * 8 + k]; s.dl5[k] = t.dl5[im * 8 + k]; s.dl6[k] = t.dl6[im * 8 + k];
        }
        s.ismono[0] = t.sig_ismonotone[im];
        s.ismono[1] = t.sig_ismonotone[nmed + im];
        s.meke = m.meke;
        for (int j = 0; j < D_MXGE; j++) {
            size_t o = (size_t)im * D_MXGE + j;
            PhBin<R> &b = L.ph[o];
            b.gmfp = mkpl<R>(t.gmfp1[o], t.gmfp0[o]);
            b.cohe = mkpl<R>(t.cohe1[o], t.cohe0[o]);
            b.gbr1 = mkpl<R>(t.gbr11[o], t.gbr10[o]);
            b.gbr2 = mkpl<R>(t.gbr21[o], t.gbr20[o]);
            L.pmax[o] = mkpl<R>(t.pmax1[o], t.pmax0[o]);
        }
        for (int j = 0; j < D_MXRAYFF; j++) {
            size_t o = (size_t)im * D_MXRAYFF + j;
            L.ray[im].xgrid[j] = t.xgrid[o];
            L.ray[im].fcum[j] = t.fcum[o];
            L.ray[im].b[j] = t.b_array[o];
            L.ray[im].c[j] = t.c_array[o];
            L.ray[im].ia[j] = t.i_array[o];
        }
        for (int q = 0; q < 2; q++)
            for (int j = 0; j < D_MXEKE; j++) {
                size_t o = (size_t)im * D_MXEKE + j;
                ElBin<R> &b = L.el[((size_t)im * 2 + q) * D_MXEKE + j];
                if (q == 0) {
                    b.sig = mkpl<R>(t.esig1[o], t.esig0[o]);
                    b.dedx = mkpl<R>(t.ededx1[o], t.ededx0[o]);
                    b.eta = mkpl<R>(t.etae_ms1[o], t.etae_ms0[o]);
                    b.q1c = mkpl<R>(t.q1ce_ms1[o], t.q1ce_ms0[o]);
                    b.q2c = mkpl<R>(t.q2ce_ms1[o], t.q2ce_ms0[o]);
                    b.br1 = mkpl<R>(t.ebr11[o], t.ebr10[o]);
                    b.br2 = mkpl<R>(0.0, 0.0);
                } else {
                    b.sig = mkpl<R>(t.psig1[o], t.psig0[o]);
                    b.dedx = mkpl<R>(t.pdedx1[o], t.pdedx0[o]);
                    b.eta = mkpl<R>(t.etap_ms1[o], t.etap_ms0[o]);
                    b.q1c = mkpl<R>(t.q1cp_ms1[o], t.q1cp_ms0[o]);
                    b.q2c = mkpl<R>(t.q2cp_ms1[o], t.q2cp_ms0[o]);
                    b.br1 = mkpl<R>(t.pbr11[o], t.pbr10[o]);
                    b.br2 = mkpl<R>(t.pbr21[o], t.pbr20[o]);
                }
                b.tmxs = mkpl<R>(t.tmxs1[o], t.tmxs0[o]);
                b.blcce = mkpl<R>(t.blcce1[o], t.blcce0[o]);
                b.range = (R)t.range_ep[(size_t)q * nmed * D_MXEKE + o];
                b.earr = (R)t.e_array[o];
            }
    }
    L.msurf.assign(D_NMS, MsE<R>{});
    for (int i = 0; i < D_NMS; i++) {
        L.msurf[i].u = (R)t.ums[i];
        L.msurf[i].f = (R)t.fms[i];
        L.msurf[i].w = (R)t.wms[i];
        L.msurf[i].i = t.ims[i];
    }
    L.spin.assign(t.spin_rej.begin(), t.spin_rej.end());
    d.b2spin_min = t.b2spin_min; d.dbeta2i = t.dbeta2i; d.espml = t.espml; d.dleneri = t.dleneri;
    d.dqq1i = t.dqq1i; d.dllambi = t.dllambi; d.dqmsi = t.dqmsi;
}
template void make_layout<double>(const Tables &, const Phantom &, const Regions &, double, double, int,
                                  Layout<double> &);
template void make_layout<float>(const Tables &, const Phantom &, const Regions &, double, double, int,
                                 Layout<float> &);

template <typename R>
void point_layout_at_host(Layout<R> &L) {
    DevData<R> &d = L.d;
    d.xb = L.xb.data(); d.yb = L.yb.data(); d.zb = L.zb.data();
    d.med = L.med.data(); d.rhof = L.rhof.data();
    d.ms = L.ms.data(); d.ph = L.ph.data(); d.pmax = L.pmax.data(); d.ray = L.ray.data(); d.el = L.el.data();
    d.msurf = L.msurf.data(); d.spin = L.spin.data();
}
template void point_layout_at_host<double>(Layout<double> &);
template void point_layout_at_host<float>(Layout<float> &);

template <typename R>
static int build_devset(omc_engine *e, DevSet<R> &S) {
    Layout<R> L;
    make_layout<R>(e->tabs, e->ph, e->reg, e->opt.ecut, e->opt.pcut, e->opt.ref_compat, L);
    int rc;
    if ((rc = upload(e, S.xb, L.xb))) return rc;
    if ((rc = upload(e, S.yb, L.yb))) return rc;
    if ((rc = upload(e, S.zb, L.zb))) return rc;
    if ((rc = upload(e, S.med, L.med))) return rc;
    if ((rc = upload(e, S.rhof, L.rhof))) return rc;
    if ((rc = upload(e, S.ms, L.ms))) return rc;
    if ((rc = upload(e, S.ph, L.ph))) return rc;
    if ((rc = upload(e, S.pmax, L.pmax))) return rc;
    if ((rc = upload(e, S.ray, L.ray))) return rc;
    if ((rc = upload(e, S.el, L.el))) return rc;
    if ((rc = upload(e, S.msurf, L.msurf))) return rc;
    if ((rc = upload(e, S.spin, L.spin))) return rc;
    S.d = L.d;
    DevData<R> &d = S.d;
    d.nsplit = e->opt.nsplit > 1 ? e->opt.nsplit : 1;
    // the plain FP64 form keeps the reference's per-step restart (its
    // trajectories replay the reference's); the event form re-draws after
    // electron_chsteps steps
    d.chsteps = sizeof(R) == 4 ? std::max(0, e->opt.electron_chsteps) : 0;
    d.defer_interact = sizeof(R) == 4 ? (e->opt.electron_interact_kernel ? 1 : 0) : 0;
    d.woodcock = sizeof(R) == 4 && d.uniform && e->opt.photon_woodcock ? 1 : 0;
    d.xb = S.xb.template as<R>(); d.yb = S.yb.template as<R>(); d.zb = S.zb.template as<R>();
    d.med = S.med.template as<int8_t>(); d.rhof = S.rhof.template as<R>();
    d.ms = S.ms.template as<MedS<R>>(); d.ph = S.ph.template as<PhBin<R>>(); d.pmax = S.pmax.template as<PL<R>>();
    d.ray = S.ray.template as<Rayl<R>>(); d.el = S.el.template as<ElBin<R>>();
    d.msurf = S.msurf.template as<MsE<R>>(); d.spin = S.spin.template as<R>();
    return OMC_OK;
}

// ------------------------------------------------------ batch statistics
// Sum and sum of squares of the batch tallies, then zero the working tally
// (accumEndep, omc_dosxyz.c:696-717; the matRad variant scales each batch
// by 1/nperbatch, omc_matrad.c:897-918).  One pass, HBM-bound: the working
// tally is read once and written with zeros, the accumulators read+written.
__global__ void k_fold(double *__restrict__ work, double *__restrict__ sum, double *__restrict__ sum2, long n,
                       double scale) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double x = work[i] * scale;
        sum[i] += x;
        sum2[i] += x * x;
        work[i] = 0.0;
    }
}

// dosxyz: dose in Gy per history and batch-method relative uncertainty
// (accumulateResults, omc_dosxyz.c:719-799).
__global__ void k_finalize_dosxyz(const double *sum, const double *sum2, const double *mass, const double *rho,
                                  long n, int nbatch, double nper, double *dose, double *unc) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double en = sum[i] / (double)nbatch;
        double en2 = sum2[i] / (double)nbatch;
        double u;
        if (en != 0.0) {
            u = en2 - en * en;
            u /= (double)(nbatch - 1);
            u = sqrt(u) / en;
        } else {
            en = 0.0;
            u = 0.9999999;
        }
        en *= 1.602E-10 / (mass[i] * nper);
        if (rho[i] < 0.044) {
            en = 0.0;
            u = 0.9999999;
        }
        dose[i] = en;
        unc[i] = u;
    }
}

// matRad: dose per history and variance of the mean (accumulateResults,
// omc_matrad.c:920-1012).
__global__ void k_finalize_matrad(const double *sum, const double *sum2, const double *mass, const double *rho, long n,
                                  int nbatch, double *dose, double *var) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double f = 1.602E-10 / mass[i];
        double en = sum[i] * f, en2 = sum2[i] * f * f;
        en /= (double)nbatch;
        en2 /= (double)(nbatch - 1);
        double u;
        if (en != 0.0) {
            u = en2 - en * en;
            u /= nbatch;
        } else {
            en = 0.0;
            u = 0.0;
        }
        if (rho[i] < 0.044) {
            en = 0.0;
            u = 0.0;
        }
        dose[i] = en;
        var[i] = u;
    }
}

__global__ void k_sum(const double *x, long n, double *out) {
    double s = 0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) s += x[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

int fold(omc_engine *e, double *work, double *sum, double *sum2, long n, double scale) {
    int g = std::max(1, std::min((int)((n + 255) / 256), e->sm_count * 8));
    k_fold<<<g, 256, 0, e->stream>>>(work, sum, sum2, n, scale);
    return cuda_check(e, cudaGetLastError(), "k_fold");
}

int finalize_dosxyz(omc_engine *e, const double *sum, const double *sum2, int nbatch, double nper, double *dose,
                    double *unc) {
    long n = e->ph.nvox();
    int g = std::max(1, std::min((int)((n + 255) / 256), e->sm_count * 8));
    k_finalize_dosxyz<<<g, 256, 0, e->stream>>>(sum, sum2, e->mass_d.as<double>(), e->rho_vox.as<double>(), n, nbatch,
                                                nper, dose, unc);
    return cuda_check(e, cudaGetLastError(), "k_finalize_dosxyz");
}

int finalize_matrad(omc_engine *e, const double *sum, const double *sum2, int nbatch, double *dose, double *var) {
    long n = e->ph.nvox();
    int g = std::max(1, std::min((int)((n + 255) / 256), e->sm_count * 8));
    k_finalize_matrad<<<g, 256, 0, e->stream>>>(sum, sum2, e->mass_d.as<double>(), e->rho_vox.as<double>(), n, nbatch,
                                                dose, var);
    return cuda_check(e, cudaGetLastError(), "k_finalize_matrad");
}

int device_sum(omc_engine *e, const double *x, long n, double *out_d) {
    int g = std::max(1, std::min((int)((n + 255) / 256), e->sm_count * 4));
    k_sum<<<g, 256, 0, e->stream>>>(x, n, out_d);
    return cuda_check(e, cudaGetLastError(), "k_sum");
}

// Collimator set-up of the beam source (initSource, omc_dosxyz.c:521-593).
template <typename R>
BeamSrc<R> beam_setup(const omc_engine *e, const omc_beam *b) {
    const Phantom &ph = e->ph;
    BeamSrc<R> s{};
    s.charge = b->energy.charge;
    s.spectrum = b->energy.n > 0 ? 1 : 0;
    s.energy = (R)b->energy.mono_energy;
    s.deltak = (R)b->energy.n;
    s.ssd = (R)b->ssd;
    double xinl = b->xinl, xinu = b->xinu, yinl = b->yinl, yinu = b->yinu;
    auto clampc = [](double &lo, double &hi, const std::vector<double> &bd, int n) {
        if (lo < bd[0]) lo = bd[0];
        if (hi <= lo) hi = lo;
        if (hi > bd[n]) hi = bd[n];
        if (lo > bd[n]) lo = bd[n];
    };
    clampc(xinl, xinu, ph.xb, ph.nx);
    clampc(yinl, yinu, ph.yb, ph.ny);
    auto lowidx = [](double lo, const std::vector<double> &bd, int n) {
        int i = 0;
        while (i < n - 1 && bd[i] <= lo && bd[i + 1] < lo) i++;
        return i;
    };
    s.xinl = (R)xinl;
    s.yinl = (R)yinl;
    s.xsize = (R)(xinu - xinl);
    s.ysize = (R)(yinu - yinl);
    s.ixinl = lowidx(xinl, ph.xb, ph.nx);
    s.iyinl = lowidx(yinl, ph.yb, ph.ny);
    return s;
}
template BeamSrc<double> beam_setup<double>(const omc_engine *, const omc_beam *);
template BeamSrc<float> beam_setup<float>(const omc_engine *, const omc_beam *);

}  // namespace omc

// =================================================================== C ABI
extern "C" {

const char *omc_status_string(int s) {
    switch (s) {
        case OMC_OK: return "ok";
        case OMC_E_ARG: return "invalid argument";
        case OMC_E_IO: return "cannot open file";
        case OMC_E_FORMAT: return "malformed input";
        case OMC_E_MEDIA: return "medium not found";
        case OMC_E_RANGE: return "out of supported range";
        case OMC_E_CUDA: return "CUDA failure";
        case OMC_E_NOMEM: return "out of device memory";
        case OMC_E_DEVICE: return "device error flag";
        case OMC_E_BUSY: return "queue full";
        case OMC_E_NOTREADY: return "not ready";
        default: return "unknown status";
    }
}

const char *omc_last_error(void) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    return g_err.c_str();
}

int omc_version(void) { return 10000; }

int64_t omc_device_allocations(void) { return g_device_allocs.load(std::memory_order_relaxed); }

int omc_tables_build(const char *pegs_file, const char *pgs4form_file, const char *data_folder,
                     const char *const *media, int nmed, omc_tables **out) {
    if (!pegs_file || !pgs4form_file || !data_folder || !media || !out || nmed <= 0)
        return global_err(OMC_E_ARG, "omc_tables_build: null argument");
    *out = nullptr;
    DataPaths p{pegs_file, pgs4form_file, data_folder};
    std::vector<std::string> names;
    for (int i = 0; i < nmed; i++) {
        if (!media[i]) return global_err(OMC_E_ARG, "omc_tables_build: null medium name");
        names.push_back(strip_spaces(media[i]));
    }
    auto *t = new omc_tables();
    std::string err;
    int rc = build_tables(p, names, t->t, err);
    if (rc) {
        delete t;
        return global_err(rc, err);
    }
    *out = t;
    return OMC_OK;
}

void omc_tables_free(omc_tables *t) { delete t; }

int omc_tables_nmed(const omc_tables *t) { return t ? t->t.nmed : 0; }

int omc_tables_get(const omc_tables *tt, const char *name, const void **data, int64_t *n, int *is_int) {
    if (!tt || !name || !data || !n || !is_int) return global_err(OMC_E_ARG, "omc_tables_get: null argument");
    const Tables &t = tt->t;
    static thread_local std::vector<double> scratch;
    static thread_local std::vector<int> scratch_i;
    *is_int = 0;
#define D(NAME, VEC) if (!std::strcmp(name, NAME)) { *data = t.VEC.data(); *n = (int64_t)t.VEC.size(); return OMC_OK; }
#define I(NAME, VEC) if (!std::strcmp(name, NAME)) { *data = t.VEC.data(); *n = (int64_t)t.VEC.size(); *is_int = 1; return OMC_OK; }
    D("ge0", ge0) D("ge1", ge1) D("gmfp0", gmfp0) D("gmfp1", gmfp1) D("gbr10", gbr10) D("gbr11", gbr11)
    D("gbr20", gbr20) D("gbr21", gbr21) D("cohe0", cohe0) D("cohe1", cohe1)
    D("xgrid", xgrid) D("fcum", fcum) D("b_array", b_array) D("c_array", c_array) D("pmax0", pmax0) D("pmax1", pmax1)
    I("i_array", i_array)
    D("dl1", dl1) D("dl2", dl2) D("dl3", dl3) D("dl4", dl4) D("dl5", dl5) D("dl6", dl6)
    D("bpar0", bpar0) D("bpar1", bpar1) D("delcm", delcm) D("zbrang", zbrang)
    D("esig0", esig0) D("esig1", esig1) D("psig0", psig0) D("psig1", psig1) D("ededx0", ededx0) D("ededx1", ededx1)
    D("pdedx0", pdedx0) D("pdedx1", pdedx1) D("ebr10", ebr10) D("ebr11", ebr11) D("pbr10", pbr10) D("pbr11", pbr11)
    D("pbr20", pbr20) D("pbr21", pbr21) D("tmxs0", tmxs0) D("tmxs1", tmxs1) D("blcce0", blcce0) D("blcce1", blcce1)
    D("etae_ms0", etae_ms0) D("etae_ms1", etae_ms1) D("etap_ms0", etap_ms0) D("etap_ms1", etap_ms1)
    D("q1ce_ms0", q1ce_ms0) D("q1ce_ms1", q1ce_ms1) D("q1cp_ms0", q1cp_ms0) D("q1cp_ms1", q1cp_ms1)
    D("q2ce_ms0", q2ce_ms0) D("q2ce_ms1", q2ce_ms1) D("q2cp_ms0", q2cp_ms0) D("q2cp_ms1", q2cp_ms1)
    D("range_ep", range_ep) D("e_array", e_array) D("eke0", eke0) D("eke1", eke1) D("esig_e", esig_e)
    D("psig_e", psig_e) D("xcc", xcc) D("blcc", blcc) D("expeke1", expeke1) I("sig_ismonotone", sig_ismonotone)
    D("spin_rej", spin_rej) D("ums", ums) D("fms", fms) D("wms", wms) I("ims", ims)
#undef D
#undef I
    auto per_med = [&](auto f) {
        scratch.assign(t.nmed, 0.0);
        for (int i = 0; i < t.nmed; i++) scratch[i] = f(t.pegs[i]);
        *data = scratch.data();
        *n = t.nmed;
        return OMC_OK;
    };
    if (!std::strcmp(name, "rho")) return per_med([](const PegsMedium &m) { return m.rho; });
    if (!std::strcmp(name, "rlc")) return per_med([](const PegsMedium &m) { return m.rlc; });
    if (!std::strcmp(name, "ae")) return per_med([](const PegsMedium &m) { return m.ae; });
    if (!std::strcmp(name, "ap")) return per_med([](const PegsMedium &m) { return m.ap; });
    if (!std::strcmp(name, "ue")) return per_med([](const PegsMedium &m) { return m.ue; });
    if (!std::strcmp(name, "up")) return per_med([](const PegsMedium &m) { return m.up; });
    if (!std::strcmp(name, "te")) return per_med([](const PegsMedium &m) { return m.te; });
    if (!std::strcmp(name, "thmoll")) return per_med([](const PegsMedium &m) { return m.thmoll; });
    if (!std::strcmp(name, "meke")) {
        scratch_i.assign(t.nmed, 0);
        for (int i = 0; i < t.nmed; i++) scratch_i[i] = t.pegs[i].meke;
        *data = scratch_i.data();
        *n = t.nmed;
        *is_int = 1;
        return OMC_OK;
    }
    if (!std::strcmp(name, "spin_scalars")) {
        scratch = {t.b2spin_min, t.dbeta2i, t.espml, t.dleneri, t.dqq1i, t.dllambi, t.dqmsi};
        *data = scratch.data();
        *n = 7;
        return OMC_OK;
    }
    return global_err(OMC_E_ARG, std::string("unknown table: ") + name);
}

int omc_spectrum_load(const char *path, double *cdf1, double *cdf2, int *n) {
    if (!path || !cdf1 || !cdf2 || !n) return global_err(OMC_E_ARG, "omc_spectrum_load: null argument");
    Spectrum s;
    std::string err;
    int rc = read_spectrum(path, s, err);
    if (rc) return global_err(rc, err);
    std::copy(s.cdfinv1.begin(), s.cdfinv1.end(), cdf1);
    std::copy(s.cdfinv2.begin(), s.cdfinv2.end(), cdf2);
    *n = (int)s.cdfinv1.size();
    return OMC_OK;
}

void omc_options_default(omc_options *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->ecut = 0.7;
    o->pcut = 0.01;
    o->device = 0;
    o->ref_compat = 1;
    o->queue_capacity = 0;
    o->block = 0;
    o->nsplit = 1;
    o->electron_split = 0.0;
    o->electron_chsteps = 3;
    o->electron_interact_kernel = 1;
    o->photon_woodcock = 1;
}

int omc_engine_create(const omc_tables *t, const omc_phantom *ph, const omc_options *o, omc_engine **out) {
    if (!t || !ph || !out) return global_err(OMC_E_ARG, "omc_engine_create: null argument");
    *out = nullptr;
    if (ph->nx <= 0 || ph->ny <= 0 || ph->nz <= 0 || !ph->xb || !ph->yb || !ph->zb || !ph->med || !ph->rho)
        return global_err(OMC_E_ARG, "omc_engine_create: incomplete phantom");
    omc_options opt;
    omc_options_default(&opt);
    if (o) opt = *o;
    if (opt.nsplit < 1) return global_err(OMC_E_ARG, "nsplit must be >= 1");
    if (opt.nsplit > OMC_MAX_NSPLIT)
        return global_err(OMC_E_RANGE, "nsplit above " + std::to_string(OMC_MAX_NSPLIT) + " is not supported");
    int ndev = 0;
    cudaError_t cr = cudaGetDeviceCount(&ndev);
    if (cr != cudaSuccess || ndev == 0)
        return global_err(OMC_E_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(cr));
    if (opt.device < 0 || opt.device >= ndev) return global_err(OMC_E_ARG, "device ordinal out of range");
    auto *e = new omc_engine();
    e->opt = opt;
    e->device = opt.device;
    e->tabs = t->t;
    Phantom &P = e->ph;
    P.nx = ph->nx; P.ny = ph->ny; P.nz = ph->nz;
    P.xb.assign(ph->xb, ph->xb + ph->nx + 1);
    P.yb.assign(ph->yb, ph->yb + ph->ny + 1);
    P.zb.assign(ph->zb, ph->zb + ph->nz + 1);
    long nv = P.nvox();
    P.med.assign(ph->med, ph->med + nv);
    P.rho.assign(ph->rho, ph->rho + nv);
    std::string err;
    int rc = build_regions(P, e->tabs, opt.ecut, opt.pcut, e->reg, err);
    if (rc) {
        delete e;
        return global_err(rc, err);
    }
    auto fail = [&](int code) {
        std::string m = e->err;
        delete e;
        return global_err(code, m);
    };
    if ((rc = cuda_check(e, cudaSetDevice(e->device), "cudaSetDevice"))) return fail(rc);
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, e->device);
    e->sm_count = prop.multiProcessorCount;
    if ((rc = cuda_check(e, cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking), "stream"))) return fail(rc);
    if ((rc = build_devset<double>(e, e->d64))) return fail(rc);
    if ((rc = build_devset<float>(e, e->d32))) return fail(rc);
    e->mass.resize(nv);
    for (long v = 0; v < nv; v++) {
        int i = v % P.nx, j = (v / P.nx) % P.ny, k = v / ((long)P.nx * P.ny);
        e->mass[v] = (P.xb[i + 1] - P.xb[i]) * (P.yb[j + 1] - P.yb[j]) * (P.zb[k + 1] - P.zb[k]) * P.rho[v];
    }
    if ((rc = upload(e, e->mass_d, e->mass))) return fail(rc);
    if ((rc = upload(e, e->rho_vox, P.rho))) return fail(rc);
    if ((rc = e->errword.alloc(sizeof(unsigned)))) return fail(set_err(e, rc, "alloc"));
    cudaMemset(e->errword.p, 0, sizeof(unsigned));
    *out = e;
    return OMC_OK;
}

int omc_engine_destroy(omc_engine *e) {
    if (!e) return OMC_OK;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    event_release(e);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return OMC_OK;
}

const char *omc_engine_last_error(const omc_engine *e) { return e ? e->err.c_str() : omc_last_error(); }

int omc_event_params(omc_engine *e, int electron_tsteps, int tail_boost, int64_t inflight, int block,
                     double electron_split, int electron_chsteps, int64_t drain_particles) {
    if (!e) return global_err(OMC_E_ARG, "omc_event_params: null engine");
    cudaSetDevice(e->device);
    if (drain_particles >= -1) e->opt.drain_particles = drain_particles;
    if (electron_chsteps >= 0) {
        e->opt.electron_chsteps = electron_chsteps;
        e->d32.d.chsteps = electron_chsteps;
    }
    return event_set_params(e, electron_tsteps, tail_boost, (long long)inflight, block, electron_split);
}

int omc_profile_last(const omc_engine *e, double *out, int n) {
    if (!e || !out || n < 28) return global_err(OMC_E_ARG, "omc_profile_last: bad argument");
    for (int i = 0; i < 28; i++) out[i] = 0;
    if (!e->ev) return OMC_OK;
    for (int k = 0; k < 4; k++) {
        const KernelProfile &P = e->ev->prof[k];
        double v[7] = {P.launches, P.seconds, P.particles, P.steps, P.cross, P.dep, P.atom};
        for (int j = 0; j < 7; j++) out[k * 7 + j] = v[j];
    }
    return OMC_OK;
}

int omc_profile_drain(const omc_engine *e, double *out, int n) {
    if (!e || !out || n < 5) return global_err(OMC_E_ARG, "omc_profile_drain: bad argument");
    for (int i = 0; i < 5; i++) out[i] = e->ev ? e->ev->drain_stats[i] : 0.0;
    return OMC_OK;
}

int omc_profile_trace(const omc_engine *e, double *out, int max_cycles) {
    if (!e || (max_cycles > 0 && !out)) return global_err(OMC_E_ARG, "omc_profile_trace: bad argument");
    if (!e->ev) return 0;
    const std::vector<double> &t = e->ev->trace;
    int n = (int)(t.size() / 6);
    int m = std::min(n, std::max(max_cycles, 0));
    std::copy(t.begin(), t.begin() + (size_t)m * 6, out);
    return n;
}

// ------------------------------------------------------------ beam runs
int omc_run_beam(omc_engine *e, const omc_beam *b, int64_t ncase, int nbatch, uint64_t seed, int mode, double *dose,
                 double *unc, double *stats) {
    if (!e || !b) return global_err(OMC_E_ARG, "omc_run_beam: null argument");
    if (nbatch < 2) return set_err(e, OMC_E_ARG, "nbatch must be >= 2 for the batch uncertainty");
    if (mode != OMC_PLAIN_FP64 && mode != OMC_EVENT_FP32 && mode != OMC_EVENT_FP64)
        return set_err(e, OMC_E_ARG, "unknown mode");
    if (b->energy.n > 0 && (!b->energy.cdf1 || !b->energy.cdf2)) return set_err(e, OMC_E_ARG, "spectrum arrays missing");
    if (b->energy.charge < -1 || b->energy.charge > 1) return set_err(e, OMC_E_ARG, "charge must be -1, 0 or 1");
    cudaSetDevice(e->device);
    // ncase -> nperbatch * nbatch (omc_dosxyz.c:1222-1229)
    if (ncase / nbatch == 0) ncase = nbatch;
    long nper = (long)(ncase / nbatch);
    long nv = e->ph.nvox();
    int rc;
    DBuf &sum = e->run_sum, &sum2 = e->run_sum2, &out_d = e->run_out, &unc_d = e->run_unc, &cdf = e->run_cdf,
         &acc = e->run_acc;
    if ((rc = sum.reserve(nv * 8)) || (rc = sum2.reserve(nv * 8)) || (rc = out_d.reserve(nv * 8)) ||
        (rc = unc_d.reserve(nv * 8)) || (rc = acc.reserve(4 * 8)))
        return set_err(e, rc, "device allocation for tallies failed");
    cudaMemsetAsync(sum.p, 0, nv * 8, e->stream);
    cudaMemsetAsync(sum2.p, 0, nv * 8, e->stream);
    cudaMemsetAsync(acc.p, 0, 4 * 8, e->stream);
    cudaMemsetAsync(e->errword.p, 0, sizeof(unsigned), e->stream);
    int ncdf = b->energy.n;
    KernelStats ks;
    if (mode == OMC_PLAIN_FP64) {
        std::vector<double> c;
        if (ncdf > 0) {
            c.assign(b->energy.cdf1, b->energy.cdf1 + ncdf);
            c.insert(c.end(), b->energy.cdf2, b->energy.cdf2 + ncdf);
            if ((rc = cdf.reserve(c.size() * 8))) return set_err(e, rc, "device allocation failed");
            cudaMemcpyAsync(cdf.p, c.data(), c.size() * 8, cudaMemcpyHostToDevice, e->stream);
        }
        BeamSrc<double> S = beam_setup<double>(e, b);
        S.cdf1 = ncdf > 0 ? cdf.as<double>() : nullptr;
        S.cdf2 = ncdf > 0 ? cdf.as<double>() + ncdf : nullptr;
        DBuf &work = e->run_work;
        if ((rc = work.reserve(nv * 8))) return set_err(e, rc, "device allocation for tallies failed");
        cudaMemsetAsync(work.p, 0, nv * 8, e->stream);
        int block = e->opt.block > 0 ? e->opt.block : 128;
        cudaEvent_t t0, t1;
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, e->stream);
        for (int ib = 0; ib < nbatch; ib++) {
            long nl = 0;
            if ((rc = plain_beam_batch(e, S, work.as<double>(), seed, (long)ib * nper, nper, acc.as<double>() + 1,
                                       block, &nl)))
                return rc;
            if ((rc = fold(e, work.as<double>(), sum.as<double>(), sum2.as<double>(), nv, 1.0))) return rc;
            ks.launches += nl + 1;
        }
        cudaEventRecord(t1, e->stream);
        if ((rc = cuda_check(e, cudaEventSynchronize(t1), "beam transport"))) return rc;
        float ms = 0;
        cudaEventElapsedTime(&ms, t0, t1);
        ks.seconds = ms * 1e-3;
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
    } else {
        auto run = mode == OMC_EVENT_FP64 ? event_run_beam<double> : event_run_beam<float>;
        if ((rc = run(e, b, nper, nbatch, seed, sum.as<double>(), sum2.as<double>(), acc.as<double>() + 1,
                                 ks)))
            return rc;
    }
    if ((rc = device_sum(e, sum.as<double>(), nv, acc.as<double>()))) return rc;
    if ((rc = finalize_dosxyz(e, sum.as<double>(), sum2.as<double>(), nbatch, (double)nper, out_d.as<double>(),
                              unc_d.as<double>())))
        return rc;
    double accum[4];
    unsigned flags = 0;
    if ((rc = cuda_check(e, cudaMemcpyAsync(accum, acc.p, 4 * 8, cudaMemcpyDeviceToHost, e->stream), "d2h"))) return rc;
    cudaMemcpyAsync(&flags, e->errword.p, sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream);
    if (dose) cudaMemcpyAsync(dose, out_d.p, nv * 8, cudaMemcpyDeviceToHost, e->stream);
    if (unc) cudaMemcpyAsync(unc, unc_d.p, nv * 8, cudaMemcpyDeviceToHost, e->stream);
    if ((rc = cuda_check(e, cudaStreamSynchronize(e->stream), "beam results"))) return rc;
    ks.flags |= flags;
    if (stats) {
        stats[0] = (double)nper * nbatch;
        stats[1] = ks.seconds;
        stats[2] = (double)ks.launches;
        stats[3] = accum[0];
        stats[4] = accum[1];
        stats[5] = (double)ks.flags;
    }
    if (ks.flags & (ERR_STACK | ERR_QUEUE | ERR_NAN))
        return set_err(e, OMC_E_DEVICE, "device error flags " + std::to_string(ks.flags) + " (particles dropped)");
    return OMC_OK;
}

// ------------------------------------------------------- validation hooks
int omc_trace_rays(omc_engine *e, const double *rays, int nrays, int cap, double *ustep, int32_t *irnew,
                   int32_t *idisc, int32_t *ncalls, double *hownear_out) {
    if (!e || !rays || nrays <= 0 || cap <= 0 || !ustep || !irnew || !idisc || !ncalls)
        return global_err(OMC_E_ARG, "omc_trace_rays: bad argument");
    cudaSetDevice(e->device);
    DBuf r, us, irn, idc, nc, hn;
    int rc;
    long m = (long)nrays * cap;
    if ((rc = r.alloc(nrays * 7 * 8)) || (rc = us.alloc(m * 8)) || (rc = irn.alloc(m * 4)) || (rc = idc.alloc(m * 4)) ||
        (rc = nc.alloc(nrays * 4)) || (rc = hn.alloc(nrays * 8)))
        return set_err(e, rc, "alloc");
    cudaMemcpyAsync(r.p, rays, nrays * 7 * 8, cudaMemcpyHostToDevice, e->stream);
    if ((rc = plain_trace(e, r.as<double>(), nrays, cap, us.as<double>(), irn.as<int>(), idc.as<int>(), nc.as<int>(),
                          hn.as<double>())))
        return rc;
    cudaMemcpyAsync(ustep, us.p, m * 8, cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(irnew, irn.p, m * 4, cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(idisc, idc.p, m * 4, cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(ncalls, nc.p, nrays * 4, cudaMemcpyDeviceToHost, e->stream);
    if (hownear_out) cudaMemcpyAsync(hownear_out, hn.p, nrays * 8, cudaMemcpyDeviceToHost, e->stream);
    return cuda_check(e, cudaStreamSynchronize(e->stream), "omc_trace_rays");
}

int omc_replay(omc_engine *e, const double *prim, int nhist, const double *rn, const int64_t *rn_off, int dep_cap,
               int32_t *dep_ir, double *dep_e, int32_t *ndep, int64_t *nused, uint32_t *flags) {
    if (!e || !prim || nhist <= 0 || !rn || !rn_off || dep_cap <= 0 || !dep_ir || !dep_e || !ndep || !nused || !flags)
        return global_err(OMC_E_ARG, "omc_replay: bad argument");
    cudaSetDevice(e->device);
    long nrn = rn_off[nhist];
    long m = (long)nhist * dep_cap;
    DBuf pd, rd, od, di, de, nd, nu, fl, sk;
    int rc;
    if ((rc = pd.alloc(nhist * 11 * 8)) || (rc = rd.alloc(std::max(1L, nrn) * 8)) || (rc = od.alloc((nhist + 1) * 8)) ||
        (rc = di.alloc(m * 4)) || (rc = de.alloc(m * 8)) || (rc = nd.alloc(nhist * 4)) || (rc = nu.alloc(nhist * 8)) ||
        (rc = fl.alloc(nhist * 4)) || (rc = sk.alloc(plain_replay_stack_bytes(nhist))))
        return set_err(e, rc, "alloc");
    cudaMemcpyAsync(pd.p, prim, nhist * 11 * 8, cudaMemcpyHostToDevice, e->stream);
    if (nrn > 0) cudaMemcpyAsync(rd.p, rn, nrn * 8, cudaMemcpyHostToDevice, e->stream);
    cudaMemcpyAsync(od.p, rn_off, (nhist + 1) * 8, cudaMemcpyHostToDevice, e->stream);
    if ((rc = plain_replay(e, pd.as<double>(), nhist, rd.as<double>(), od.as<long>(), dep_cap, di.as<int>(),
                           de.as<double>(), nd.as<int>(), nu.as<long>(), fl.as<unsigned>(), sk.p)))
        return rc;
    cudaMemcpyAsync(dep_ir, di.p, m * 4, cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(dep_e, de.p, m * 8, cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(ndep, nd.p, nhist * 4, cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(nused, nu.p, nhist * 8, cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(flags, fl.p, nhist * 4, cudaMemcpyDeviceToHost, e->stream);
    return cuda_check(e, cudaStreamSynchronize(e->stream), "omc_replay");
}

int omc_kat(omc_engine *e, int which, const double *q, const double *extra, int n, const double *rn,
            const int64_t *rn_off, double *out, int32_t *nout, int64_t *used, uint32_t *flags) {
    if (!e || !q || n <= 0 || !rn || !rn_off || !out || !nout || !used || !flags || which < 0 || which > KAT_MSDIST ||
        (which == KAT_MSDIST && !extra))
        return global_err(OMC_E_ARG, "omc_kat: bad argument");
    cudaSetDevice(e->device);
    const long nvox = e->ph.nvox();
    for (int c = 0; c < n; c++)
        if (q[11 * c + 8] < 1 || q[11 * c + 8] > nvox) return set_err(e, OMC_E_ARG, "omc_kat: region out of range");
    long nrn = rn_off[n];
    DBuf qd, xd, rd, od, outd, nd, ud, fd;
    int rc;
    if ((rc = qd.alloc((size_t)n * 11 * 8)) || (rc = xd.alloc((size_t)n * 2 * 8)) ||
        (rc = rd.alloc(std::max(1L, nrn) * 8)) || (rc = od.alloc((size_t)(n + 1) * 8)) ||
        (rc = outd.alloc((size_t)n * KAT_MAXOUT * 11 * 8)) || (rc = nd.alloc((size_t)n * 4)) ||
        (rc = ud.alloc((size_t)n * 8)) || (rc = fd.alloc((size_t)n * 4)))
        return set_err(e, rc, "alloc");
    cudaMemcpyAsync(qd.p, q, (size_t)n * 11 * 8, cudaMemcpyHostToDevice, e->stream);
    if (extra) cudaMemcpyAsync(xd.p, extra, (size_t)n * 2 * 8, cudaMemcpyHostToDevice, e->stream);
    if (nrn > 0) cudaMemcpyAsync(rd.p, rn, nrn * 8, cudaMemcpyHostToDevice, e->stream);
    cudaMemcpyAsync(od.p, rn_off, (size_t)(n + 1) * 8, cudaMemcpyHostToDevice, e->stream);
    if ((rc = plain_kat(e, which, qd.as<double>(), xd.as<double>(), n, rd.as<double>(), od.as<long>(),
                        outd.as<double>(), nd.as<int>(), ud.as<long>(), fd.as<unsigned>())))
        return rc;
    cudaMemcpyAsync(out, outd.p, (size_t)n * KAT_MAXOUT * 11 * 8, cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(nout, nd.p, (size_t)n * 4, cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(used, ud.p, (size_t)n * 8, cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(flags, fd.p, (size_t)n * 4, cudaMemcpyDeviceToHost, e->stream);
    return cuda_check(e, cudaStreamSynchronize(e->stream), "omc_kat");
}

}  // extern "C"
