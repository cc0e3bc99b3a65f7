// Internal engine state shared by the translation units of libomcgpu.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "omc_device.cuh"
#include "omc_host.h"
#include "../../include/omcgpu.h"

struct omc_tables {
    omc::Tables t;
};

namespace omc {

// Device allocation with ownership.
struct DBuf {
    void *p = nullptr;
    size_t n = 0;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    int alloc(size_t bytes);
    // keep the buffer if it holds `bytes` already, else reallocate
    int reserve(size_t bytes) { return (p && n >= bytes) ? 0 : alloc(bytes); }
    template <typename T>
    T *as() const { return (T *)p; }
};

// One precision's worth of resident device tables and geometry.
template <typename R>
struct DevSet {
    DBuf xb, yb, zb, med, rhof, ms, ph, pmax, ray, el, msurf, spin;
    DevData<R> d{};
};

// Host image of the device layout (built once, then uploaded).
template <typename R>
struct Layout {
    std::vector<R> xb, yb, zb, rhof, spin;
    std::vector<int8_t> med;
    std::vector<MedS<R>> ms;
    std::vector<PhBin<R>> ph;
    std::vector<PL<R>> pmax;
    std::vector<Rayl<R>> ray;
    std::vector<ElBin<R>> el;
    std::vector<MsE<R>> msurf;
    DevData<R> d{};
};
template <typename R>
void make_layout(const Tables &t, const Phantom &ph, const Regions &rg, double ecut, double pcut, int ref_compat,
                 Layout<R> &L);
template <typename R>
void point_layout_at_host(Layout<R> &L);

struct KernelStats {
    double seconds = 0;     // device time of the transport kernels
    long launches = 0;      // kernel launches in the transport
    unsigned flags = 0;     // DevErr bits
};

}  // namespace omc

namespace omc {
template <typename R>
struct EventStateT;
using EventState = EventStateT<float>;
}

struct omc_engine {
    omc::EventState *ev = nullptr;  // event-form queues (allocated on first use)
    omc::EventStateT<double> *ev64 = nullptr;  // the FP64 event form's (allocated on first use)
    omc::Tables tabs;
    omc::Phantom ph;
    omc::Regions reg;
    omc_options opt{};
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    omc::DevSet<double> d64;
    omc::DevSet<float> d32;
    omc::DBuf rho_vox;      // FP64 density per voxel (dose conversion)
    omc::DBuf errword;      // unsigned device error flags
    std::string err;
    std::vector<double> mass;  // voxel mass (g), host copy
    omc::DBuf mass_d;
    // device buffers of omc_run_beam, kept between calls and grown on
    // demand so that a run allocates nothing once the engine is warm
    omc::DBuf run_sum, run_sum2, run_out, run_unc, run_acc, run_cdf, run_work, run_tal, run_cdf32;
};

namespace omc {
int set_err(omc_engine *e, int code, const std::string &msg);
int cuda_check(omc_engine *e, cudaError_t rc, const char *what);

// Plain FP64 form (omc_plain.cu).
// *launches (may be null) receives the kernel launches made: a batch is
// split into launches of at most a few million histories.
int plain_beam_batch(omc_engine *e, const BeamSrc<double> &S, double *work, uint64_t seed, long hist0, long n,
                     double *src_energy, int block, long *launches = nullptr);
int plain_beamlet_batch(omc_engine *e, const BeamletSrc<double> &S, int ib, double *work, uint64_t seed, long hist0,
                        long n, int block);
int plain_trace(omc_engine *e, const double *rays_d, int nrays, int cap, double *ustep, int *irnew, int *idisc,
                int *ncalls, double *hn);
// `stacks`: plain_replay_stack_bytes(nhist) of device memory for the
// histories' particle stacks.
size_t plain_replay_stack_bytes(int nhist);
int plain_replay(omc_engine *e, const double *prim, int nhist, const double *rn, const long *rn_off, int dep_cap,
                 int *dep_ir, double *dep_e, int *ndep, long *nused, unsigned *flags, void *stacks);
// Sampler known-answer hook (omc_kat): `out` holds KAT_MAXOUT particles of
// 11 doubles per case.
constexpr int KAT_MAXOUT = 4;
constexpr int KAT_MSDIST = 9;
int plain_kat(omc_engine *e, int which, const double *q, const double *extra, int n, const double *rn,
              const long *rn_off, double *out, int *nout, long *used, unsigned *flags);
}  // namespace omc
