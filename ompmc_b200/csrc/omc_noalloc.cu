// omc_run_beam_noalloc: the plain FP64 beam run for callers that must not
// allocate device memory while they run it.
//
// Why some callers cannot allocate: cudaMalloc and cudaFree synchronise the
// whole device and take an unbounded amount of time, which a latency-bound
// caller (a treatment-plan optimiser that evaluates dose inside its
// iteration loop) cannot afford; and a host application that owns the GPU's
// memory through its own pool allocator with a fixed budget (for example an
// interpreter hosting this library as an extension) may see an extra
// allocation fail at an arbitrary point.  Such callers create the engine at
// start-up, then call this entry point, which uses only memory that exists
// for the lifetime of the process.
//
// All scratch of the run lives in one file-scope device array of
// OMC_NOALLOC_MAX_VOXELS voxels' worth of tallies (about 10 MB); every GPU
// that loads the library holds it until the process exits.  Host code never
// passes the array's name to a kernel (on the host it is only a stand-in):
// the device address is taken once per device with cudaGetSymbolAddress,
// and again if that device's context has been replaced since.
#include <chrono>
#include <mutex>

#include "omc_engine.h"
#include "omc_event.h"

namespace omc {
int finalize_dosxyz(omc_engine *e, const double *sum, const double *sum2, int nbatch, double nper, double *dose,
                    double *unc);
int device_sum(omc_engine *e, const double *x, long n, double *out_d);
}  // namespace omc

using namespace omc;

namespace {

constexpr long MAXV = OMC_NOALLOC_MAX_VOXELS;
constexpr long MAXCDF = 1000;
// layout, in doubles: work | sum | sum2 | dose | unc (MAXV each) | cdf1 | cdf2 (MAXCDF each) | acc (8)
constexpr long OFF_WORK = 0, OFF_SUM = MAXV, OFF_SUM2 = 2 * MAXV, OFF_DOSE = 3 * MAXV, OFF_UNC = 4 * MAXV;
constexpr long OFF_CDF = 5 * MAXV, OFF_ACC = 5 * MAXV + 2 * MAXCDF;
constexpr long NDOUBLES = OFF_ACC + 8;

}  // namespace

// The fixed scratch: 5 * 262144 + 2008 doubles, about 10.5 MB per device.
static __device__ __align__(256) double g_noalloc_scratch[NDOUBLES];

namespace {

std::mutex g_mu;
double *g_scratch[64] = {};
void *g_scratch_ctx[64] = {};

// The driver's current context (CUcontext) through the runtime's entry-point
// lookup, so the library needs no link-time dependency on libcuda.
using CtxGetCurrent = int (*)(void **);
CtxGetCurrent ctx_get_current() {
    static CtxGetCurrent fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return (CtxGetCurrent)f;
    }();
    return fn;
}

// Device address of the scratch array on the engine's device (which is
// current), looked up on the first call made for that device and again
// whenever the device's context is not the one it was looked up in: a
// context torn down by cudaDeviceReset takes the old address with it.
int scratch_on(omc_engine *e, double **out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (e->device < 0 || e->device >= 64) return set_err(e, OMC_E_ARG, "device ordinal out of range");
    void *ctx = nullptr;
    CtxGetCurrent get = ctx_get_current();
    if (!get || get(&ctx) != 0 || !ctx) return set_err(e, OMC_E_CUDA, "no current CUDA context for the scratch lookup");
    if (!g_scratch[e->device] || g_scratch_ctx[e->device] != ctx) {
        void *p = nullptr;
        cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (rc != cudaSuccess)
            return set_err(e, OMC_E_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(rc));
        g_scratch[e->device] = (double *)p;
        g_scratch_ctx[e->device] = ctx;
    }
    *out = g_scratch[e->device];
    return OMC_OK;
}

}  // namespace

extern "C" int omc_run_beam_noalloc(omc_engine *e, const omc_beam *b, int64_t ncase, int nbatch, uint64_t seed,
                                    double *dose, double *unc, double *stats) {
    if (!e || !b) return OMC_E_ARG;
    if (nbatch < 2) return set_err(e, OMC_E_ARG, "nbatch must be >= 2 for the batch uncertainty");
    if (b->energy.n > 0 && (!b->energy.cdf1 || !b->energy.cdf2)) return set_err(e, OMC_E_ARG, "spectrum arrays missing");
    if (b->energy.charge < -1 || b->energy.charge > 1) return set_err(e, OMC_E_ARG, "charge must be -1, 0 or 1");
    if (e->opt.nsplit > 1)
        return set_err(e, OMC_E_RANGE, "omc_run_beam_noalloc: photon splitting (nsplit > 1) needs omc_run_beam");
    long nv = e->ph.nvox();
    if (nv > MAXV)
        return set_err(e, OMC_E_RANGE,
                       "omc_run_beam_noalloc: phantom has " + std::to_string(nv) + " voxels, the fixed scratch holds " +
                           std::to_string(MAXV) + " (OMC_NOALLOC_MAX_VOXELS); use omc_run_beam");
    int ncdf = b->energy.n;
    if (ncdf > MAXCDF)
        return set_err(e, OMC_E_RANGE, "omc_run_beam_noalloc: spectrum inverse CDF longer than 1000 points");
    int rc = cuda_check(e, cudaSetDevice(e->device), "cudaSetDevice");
    if (rc) return rc;
    double *s = nullptr;
    if ((rc = scratch_on(e, &s))) return rc;
    if (ncase / nbatch == 0) ncase = nbatch;
    long nper = (long)(ncase / nbatch);
    double *work = s + OFF_WORK, *sum = s + OFF_SUM, *sum2 = s + OFF_SUM2;
    double *dose_d = s + OFF_DOSE, *unc_d = s + OFF_UNC, *cdf = s + OFF_CDF, *acc = s + OFF_ACC;
    // the array keeps the previous call's contents: clear what accumulates
    if ((rc = cuda_check(e, cudaMemsetAsync(work, 0, nv * 8, e->stream), "clear scratch")) ||
        (rc = cuda_check(e, cudaMemsetAsync(sum, 0, nv * 8, e->stream), "clear scratch")) ||
        (rc = cuda_check(e, cudaMemsetAsync(sum2, 0, nv * 8, e->stream), "clear scratch")) ||
        (rc = cuda_check(e, cudaMemsetAsync(acc, 0, 8 * 8, e->stream), "clear scratch")) ||
        (rc = cuda_check(e, cudaMemsetAsync(e->errword.p, 0, sizeof(unsigned), e->stream), "clear error flags")))
        return rc;
    BeamSrc<double> S = beam_setup<double>(e, b);
    if (ncdf > 0) {
        if ((rc = cuda_check(e, cudaMemcpyAsync(cdf, b->energy.cdf1, ncdf * 8, cudaMemcpyHostToDevice, e->stream),
                             "spectrum upload")) ||
            (rc = cuda_check(e, cudaMemcpyAsync(cdf + MAXCDF, b->energy.cdf2, ncdf * 8, cudaMemcpyHostToDevice,
                                                e->stream),
                             "spectrum upload")))
            return rc;
        S.cdf1 = cdf;
        S.cdf2 = cdf + MAXCDF;
    } else {
        S.cdf1 = S.cdf2 = nullptr;
    }
    int block = e->opt.block > 0 ? e->opt.block : 128;
    auto t0 = std::chrono::steady_clock::now();
    long launches = 0;  // transport and fold launches, counted as omc_run_beam counts them
    for (int ib = 0; ib < nbatch; ib++) {
        if ((rc = plain_beam_batch(e, S, work, seed, (long)ib * nper, nper, acc + 1, block, &launches))) return rc;
        if ((rc = fold(e, work, sum, sum2, nv, 1.0))) return rc;
        launches++;
    }
    if ((rc = device_sum(e, sum, nv, acc))) return rc;
    if ((rc = finalize_dosxyz(e, sum, sum2, nbatch, (double)nper, dose_d, unc_d))) return rc;
    double a[2] = {0, 0};
    unsigned flags = 0;
    cudaMemcpyAsync(a, acc, 2 * 8, cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(&flags, e->errword.p, sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream);
    if (dose) cudaMemcpyAsync(dose, dose_d, nv * 8, cudaMemcpyDeviceToHost, e->stream);
    if (unc) cudaMemcpyAsync(unc, unc_d, nv * 8, cudaMemcpyDeviceToHost, e->stream);
    if ((rc = cuda_check(e, cudaStreamSynchronize(e->stream), "omc_run_beam_noalloc"))) return rc;
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (stats) {
        stats[0] = (double)nper * nbatch;
        stats[1] = secs;
        stats[2] = (double)launches;
        stats[3] = a[0];
        stats[4] = a[1];
        stats[5] = (double)flags;
    }
    if (flags & (ERR_STACK | ERR_QUEUE | ERR_NAN))
        return set_err(e, OMC_E_DEVICE, "device error flags " + std::to_string(flags) + " (particles dropped)");
    return OMC_OK;
}
