// Serving: continuous batching of beam and beamlet dose requests on one GPU,
// and the matRad dose-influence entry (omc_run_beamlets) built on it.
//
// Admitted requests share the event form's particle queues.  Each holds a
// device slot: a ServeReq entry, a source descriptor and nbatch FP64 working
// tallies.  Every transport cycle a planner kernel hands out injection room
// first come first served; the transport kernels keep a live-particle count
// per request.  When every admitted history is injected, nothing is pending
// and few particles are left, the drain kernel runs them to the end in one
// launch instead of the cycles' long tail.  A request is finished when all
// its histories are injected and its live count is zero; the host then
// folds its batch tallies, finalises
// dose and uncertainty (matRad: variance of the mean), extracts the sparse
// column (entries above rel_threshold * column maximum, rows ascending), frees
// the slot and admits the next pending request.  The sequential beamlet loop
// it replaces is omc_matrad.c:1576-1720.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>

#include "omc_event.h"
#include "omc_rng.cuh"
#include "omc_source.cuh"

namespace omc {
int finalize_dosxyz(omc_engine *e, const double *sum, const double *sum2, int nbatch, double nper, double *dose,
                    double *unc);
int finalize_matrad(omc_engine *e, const double *sum, const double *sum2, int nbatch, double *dose, double *var);

// ----------------------------------------------- sparse column extraction
constexpr int NSEG = 1024;

__global__ void k_dmax(const double *d, long n, unsigned long long *out) {
    double m = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        m = fmax(m, d[i]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    // dose is non-negative: the IEEE bit pattern orders like the value
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

__device__ __forceinline__ double thresh_of(const unsigned long long *dmaxbits, double rel) {
    return __longlong_as_double((long long)*dmaxbits) * rel;
}

// Entries above the threshold per contiguous segment of voxels.
__global__ void k_seg_count(const double *d, long n, long seglen, const unsigned long long *dmaxbits, double rel,
                            int *counts) {
    __shared__ int red[32];
    double t = thresh_of(dmaxbits, rel);
    long lo = (long)blockIdx.x * seglen, hi = min(n, lo + seglen);
    int c = 0;
    for (long i = lo + threadIdx.x; i < hi; i += blockDim.x) c += d[i] > t;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x < 32) {
        c = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0;
        for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
        if (threadIdx.x == 0) counts[blockIdx.x] = c;
    }
}

// Exclusive scan of the NSEG segment counts (one block of NSEG threads).
__global__ void k_seg_scan(const int *counts, int *offsets, long long *total) {
    __shared__ int s[NSEG];
    int i = threadIdx.x;
    s[i] = counts[i];
    __syncthreads();
    for (int o = 1; o < NSEG; o <<= 1) {
        int v = i >= o ? s[i - o] : 0;
        __syncthreads();
        s[i] += v;
        __syncthreads();
    }
    offsets[i] = s[i] - counts[i];
    if (i == NSEG - 1) *total = s[i];
}

// Ordered compaction: each segment writes its entries at its offset, in
// voxel order, a block-wide tile at a time.
__global__ void k_seg_write(const double *d, const double *v, long n, long seglen, const unsigned long long *dmaxbits,
                            double rel, const int *offsets, int *rows, double *vals, double *vars, long long cap) {
    __shared__ int wsum[32];
    double t = thresh_of(dmaxbits, rel);
    long lo = (long)blockIdx.x * seglen, hi = min(n, lo + seglen);
    long long base = offsets[blockIdx.x];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (long t0 = lo; t0 < hi; t0 += blockDim.x) {
        long i = t0 + threadIdx.x;
        bool keep = i < hi && d[i] > t;
        unsigned m = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) wsum[wid] = __popc(m);
        __syncthreads();
        int before = 0, tile = 0;
        for (int w = 0; w < nw; w++) {
            before += w < wid ? wsum[w] : 0;
            tile += wsum[w];
        }
        if (keep) {
            long long o = base + before + __popc(m & ((1u << lane) - 1));
            if (o < cap) {
                rows[o] = (int)i;
                vals[o] = d[i];
                if (vars) vars[o] = v[i];
            }
        }
        base += tile;
        __syncthreads();
    }
}

// Fold, finalise and (beamlets) column maximum of one finished request in
// one pass over its batch tallies: per voxel the batch values are summed in
// batch order (the order of k_fold over the batches, so the result is the
// same to the bit), the tallies are zeroed for the slot's next request, and
// dose with its uncertainty (dosxyz, accumulateResults omc_dosxyz.c:719-799)
// or variance of the mean (matRad, omc_matrad.c:920-1012) is written.
// HBM traffic: nbatch tallies read and zeroed, two outputs written.
// All of a voxel's batch values are loaded before any is zeroed, so a
// thread has up to NB loads in flight (loads and stores of the same array
// would otherwise be issued one after the other); streaming hints, since
// every value is touched once.  The kernel is bound by the loads it keeps
// in flight, so it is compiled for four resident blocks (64 registers, a
// few spilled bytes on the division's slow path): on the 128x128x96 grid
// 60 us instead of 162 us at the compiler's 86 registers and two blocks.
template <int NB>
__global__ void __launch_bounds__(256, 4)
    k_serve_finalize(double *__restrict__ tal, int nbatch, long nv, double scale, int kind,
                     const double *__restrict__ mass, const double *__restrict__ rho, double nper,
                     double *__restrict__ dose, double *__restrict__ second, unsigned long long *dmaxbits) {
    double m = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nv; i += (long)gridDim.x * blockDim.x) {
        double x[NB];
#pragma unroll
        for (int b = 0; b < NB; b++) x[b] = b < nbatch ? __ldcs(&tal[(size_t)b * nv + i]) : 0.0;
#pragma unroll
        for (int b = 0; b < NB; b++)
            if (b < nbatch) __stcs(&tal[(size_t)b * nv + i], 0.0);
        double sum = 0.0, sum2 = 0.0;
#pragma unroll
        for (int b = 0; b < NB; b++) {
            if (b < nbatch) {
                const double v = x[b] * scale;
                sum += v;
                sum2 += v * v;
            }
        }
        double en, u;
        if (kind == 0) {
            en = sum / (double)nbatch;
            double en2 = sum2 / (double)nbatch;
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
        } else {
            double f = 1.602E-10 / mass[i];
            en = sum * f;
            double en2 = sum2 * f * f;
            en /= (double)nbatch;
            en2 /= (double)(nbatch - 1);
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
            m = fmax(m, en);
        }
        __stcs(&dose[i], en);
        __stcs(&second[i], u);
    }
    if (kind != 0) {
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(dmaxbits, (unsigned long long)__double_as_longlong(m));
    }
}

}  // namespace omc

using namespace omc;

namespace {

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Device copy of a beamlet set, in FP32 for the event form and FP64 for the
// plain form.
struct PlanBuf {
    DBuf f32, f64;
    BeamletSrc<float> s32{};
    BeamletSrc<double> s64{};
};

template <typename R>
int upload_plan(omc_engine *e, const omc_beamlets *b, DBuf &buf, BeamletSrc<R> &s) {
    int nb = b->nbixels, nbeams = b->nbeams, ncdf = b->energy.n;
    size_t nr = (size_t)3 * nbeams + 9 * (size_t)nb + 2 * (size_t)ncdf;
    std::vector<R> v;
    v.reserve(nr);
    for (int i = 0; i < 3 * nbeams; i++) v.push_back((R)b->src[i]);
    for (int i = 0; i < 3 * nb; i++) v.push_back((R)b->corner[i]);
    for (int i = 0; i < 3 * nb; i++) v.push_back((R)b->side1[i]);
    for (int i = 0; i < 3 * nb; i++) v.push_back((R)b->side2[i]);
    for (int i = 0; i < ncdf; i++) v.push_back((R)b->energy.cdf1[i]);
    for (int i = 0; i < ncdf; i++) v.push_back((R)b->energy.cdf2[i]);
    size_t bytes = v.size() * sizeof(R) + (size_t)nb * 4 + 256;
    int rc = buf.alloc(bytes);
    if (rc) return set_err(e, rc, "beamlet set allocation failed");
    cudaMemcpyAsync(buf.p, v.data(), v.size() * sizeof(R), cudaMemcpyHostToDevice, e->stream);
    size_t ioff = ((v.size() * sizeof(R)) + 255) / 256 * 256;
    int *ib = (int *)((char *)buf.p + ioff);
    cudaMemcpyAsync(ib, b->ibeam, (size_t)nb * 4, cudaMemcpyHostToDevice, e->stream);
    R *p = (R *)buf.p;
    s = BeamletSrc<R>{};
    s.charge = b->energy.charge;
    s.spectrum = ncdf > 0 ? 1 : 0;
    s.gaussian = b->gaussian ? 1 : 0;
    s.energy = (R)b->energy.mono_energy;
    s.gauss_width = (R)b->gauss_width;
    s.src = p;
    s.corner = p + 3 * nbeams;
    s.side1 = p + 3 * nbeams + 3 * (size_t)nb;
    s.side2 = p + 3 * nbeams + 6 * (size_t)nb;
    s.cdf1 = ncdf > 0 ? p + 3 * nbeams + 9 * (size_t)nb : nullptr;
    s.cdf2 = ncdf > 0 ? p + 3 * nbeams + 9 * (size_t)nb + ncdf : nullptr;
    s.deltak = (R)ncdf;
    s.ibeam = ib;
    return OMC_OK;
}

int check_beamlets(omc_engine *e, const omc_beamlets *b) {
    if (!b || b->nbixels <= 0 || b->nbeams <= 0 || !b->ibeam || !b->src || !b->corner || !b->side1 || !b->side2)
        return set_err(e, OMC_E_ARG, "incomplete beamlet description");
    if (b->energy.n > 0 && (!b->energy.cdf1 || !b->energy.cdf2)) return set_err(e, OMC_E_ARG, "spectrum arrays missing");
    for (int i = 0; i < b->nbixels; i++)
        if (b->ibeam[i] < 0 || b->ibeam[i] >= b->nbeams) return set_err(e, OMC_E_ARG, "beamlet beam index out of range");
    return OMC_OK;
}

struct Request {
    int id = -1, kind = 0, slot = -1, state = 0;  // state 0 pending, 1 running, 2 done, 3 released
    long long nhist = 0, nper = 0;
    int nbatch = 0, bixel = 0;
    double rel = 0;
    const omc_beamlets *bl = nullptr;
    omc_beam beam{};
    DBuf cdf;
    double t_submit = 0, t_done = 0;
    std::vector<int32_t> rows;
    std::vector<double> vals, var, dose, unc;
    uint64_t seed = 0;
};

}  // namespace

constexpr int SERVE_NBMAX = 10;   // batches of a served request, at most

struct omc_server {
    // Guards everything below: submissions may come from any host thread
    // while one thread steps the server (a matRad-side producer beside the
    // driving loop); every omc_server_* call holds it for its duration.
    std::mutex mu;
    omc_engine *e = nullptr;
    int nbmax = SERVE_NBMAX, nslots = 0;
    long long target = 0;
    uint64_t seed = 0;
    DBuf tallies, sdbuf, fin;
    ServeDev *sd = nullptr;
    std::vector<std::unique_ptr<Request>> reqs;
    std::deque<int> pending;
    std::vector<int> slot_req;   // request id per slot, -1 free
    std::vector<int> order;      // running slots in admission order
    std::map<const omc_beamlets *, std::unique_ptr<PlanBuf>> plans;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long cycles = 0, drains = 0, launches = 0, finished = 0;
    std::vector<int> completed;  // finished since the last omc_server_completed
    cudaEvent_t t_start = nullptr, t_stop = nullptr;
    // Pipelined completion check: every step copies the request table, the
    // live counts and the queue counters into a pinned snapshot after its
    // transport work and then processes the previous step's snapshot, which
    // is ready once the previous work is, so the host never waits for the
    // work it has just queued.  A snapshot is valid for a slot only if it was
    // taken after the slot's request was admitted (slot_seq).
    struct Snap {
        ServeReq *req = nullptr;
        int *live = nullptr;
        unsigned *flags = nullptr;
        int *qc = nullptr;     // Ctl::cnt, Ctl::cnt_hi
        cudaEvent_t ev = nullptr;
        long long seq = 0;     // 0: none pending
    } snap[2];
    void *snap_host = nullptr;
    int cur = 0;
    long long seq = 0;               // snapshots taken so far
    long long drain_seq = -1;        // snapshots taken before the last drain
    std::vector<long long> slot_seq; // snapshots taken before each slot's admission
    cudaStream_t fin_stream = nullptr;  // finalisation, beside the transport
    ~omc_server() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (t_start) cudaEventDestroy(t_start);
        if (t_stop) cudaEventDestroy(t_stop);
        if (fin_stream) {
            cudaStreamSynchronize(fin_stream);
            cudaStreamDestroy(fin_stream);
        }
        for (auto &sn : snap)
            if (sn.ev) cudaEventDestroy(sn.ev);
        if (snap_host) cudaFreeHost(snap_host);
    }
    // state after the last step: particles in the queues, and whether every
    // running request had all its histories injected
    long long left = 0;
    bool injected = false;
    // finalise scratch (device): sum, sum2, dose, var | rows | vals | vars | seg counts/offsets | dmax | total
    double *f_sum = nullptr, *f_sum2 = nullptr, *f_dose = nullptr, *f_var = nullptr, *f_vals = nullptr,
           *f_vars = nullptr;
    int *f_rows = nullptr, *f_cnt = nullptr, *f_off = nullptr;
    unsigned long long *f_dmax = nullptr;
    long long *f_total = nullptr;
};

namespace {

// Fold, finalise and extract one finished request into host memory, on the
// finalisation stream (the transport work queued on the engine's stream
// goes on meanwhile; it does not touch this request's tallies, whose live
// count is zero and whose histories are all injected).
int finalize_request(omc_server *s, Request &r) {
    omc_engine *e = s->e;
    cudaStream_t st = s->fin_stream;
    long nv = e->ph.nvox();
    int rc;
    double scale = r.kind == 1 ? 1.0 / (double)r.nper : 1.0;
    s->launches += r.kind == 0 ? 1 : 4;   // fused fold + finalise (+ column extraction)
    double *tal = s->tallies.as<double>() + (size_t)r.slot * s->nbmax * nv;
    int g = std::max(1, std::min((int)((nv + 255) / 256), e->sm_count * 8));
    if (r.kind == 1) cudaMemsetAsync(s->f_dmax, 0, 8, st);
    static_assert(SERVE_NBMAX == 10, "k_serve_finalize is instantiated for the server's batch limit");
    k_serve_finalize<SERVE_NBMAX><<<g, 256, 0, st>>>(tal, r.nbatch, nv, scale, r.kind, e->mass_d.as<double>(),
                                                     e->rho_vox.as<double>(), (double)r.nper, s->f_dose, s->f_var,
                                                     s->f_dmax);
    if ((rc = cuda_check(e, cudaGetLastError(), "k_serve_finalize"))) return rc;
    if (r.kind == 0) {
        r.dose.resize(nv);
        r.unc.resize(nv);
        cudaMemcpyAsync(r.dose.data(), s->f_dose, nv * 8, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(r.unc.data(), s->f_var, nv * 8, cudaMemcpyDeviceToHost, st);
        return cuda_check(e, cudaStreamSynchronize(st), "finalize beam request");
    }
    long seglen = (nv + NSEG - 1) / NSEG;
    k_seg_count<<<NSEG, 256, 0, st>>>(s->f_dose, nv, seglen, s->f_dmax, r.rel, s->f_cnt);
    k_seg_scan<<<1, NSEG, 0, st>>>(s->f_cnt, s->f_off, s->f_total);
    k_seg_write<<<NSEG, 256, 0, st>>>(s->f_dose, s->f_var, nv, seglen, s->f_dmax, r.rel, s->f_off, s->f_rows,
                                       s->f_vals, s->f_vars, nv);
    if ((rc = cuda_check(e, cudaGetLastError(), "sparse extraction"))) return rc;
    long long nnz = 0;
    cudaMemcpyAsync(&nnz, s->f_total, 8, cudaMemcpyDeviceToHost, st);
    if ((rc = cuda_check(e, cudaStreamSynchronize(st), "sparse count"))) return rc;
    r.rows.resize(nnz);
    r.vals.resize(nnz);
    r.var.resize(nnz);
    if (nnz > 0) {
        cudaMemcpyAsync(r.rows.data(), s->f_rows, nnz * 4, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(r.vals.data(), s->f_vals, nnz * 8, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(r.var.data(), s->f_vars, nnz * 8, cudaMemcpyDeviceToHost, st);
    }
    return cuda_check(e, cudaStreamSynchronize(st), "sparse column");
}

int admit(omc_server *s) {
    omc_engine *e = s->e;
    bool changed = false;
    while (!s->pending.empty()) {
        int slot = -1;
        for (int k = 0; k < s->nslots; k++)
            if (s->slot_req[k] < 0) { slot = k; break; }
        if (slot < 0) break;
        Request &r = *s->reqs[s->pending.front()];
        s->pending.pop_front();
        r.slot = slot;
        r.state = 1;
        s->injected = false;
        s->slot_req[slot] = r.id;
        s->slot_seq[slot] = s->seq;
        s->order.push_back(slot);
        ServeReq q{};
        q.kind = r.kind;
        q.bixel = r.bixel;
        q.nhist = r.nhist;
        q.next = 0;
        q.nper = r.nper;
        q.seed = r.seed;
        cudaMemcpyAsync(&s->sd->req[slot], &q, sizeof(q), cudaMemcpyHostToDevice, e->stream);
        if (r.kind == 0) {
            BeamSrc<float> b = beam_setup<float>(e, &r.beam);
            if (r.beam.energy.n > 0) {
                b.cdf1 = r.cdf.as<float>();
                b.cdf2 = r.cdf.as<float>() + r.beam.energy.n;
            }
            cudaMemcpyAsync(&s->sd->beam[slot], &b, sizeof(b), cudaMemcpyHostToDevice, e->stream);
        } else {
            cudaMemcpyAsync(&s->sd->bl[slot], &s->plans[r.bl]->s32, sizeof(BeamletSrc<float>), cudaMemcpyHostToDevice,
                            e->stream);
        }
        cudaMemsetAsync(&s->sd->live[slot], 0, sizeof(int), e->stream);
        changed = true;
    }
    if (changed) {
        // pageable sources: the copies have taken the data when they return
        int n = (int)s->order.size();
        cudaMemcpyAsync(s->sd->order, s->order.data(), n * sizeof(int), cudaMemcpyHostToDevice, e->stream);
        cudaMemcpyAsync(&s->sd->norder, &n, sizeof(int), cudaMemcpyHostToDevice, e->stream);
        return cuda_check(e, cudaGetLastError(), "admission");
    }
    return OMC_OK;
}

}  // namespace

extern "C" {

int omc_server_create(omc_engine *e, int64_t mem_budget, int max_requests, uint64_t seed, omc_server **out) {
    if (!e || !out) return OMC_E_ARG;
    *out = nullptr;
    cudaSetDevice(e->device);
    int rc = event_prepare(e);
    if (!rc) rc = event_interact_queue(e);
    if (rc) return rc;
    auto s = std::make_unique<omc_server>();
    s->e = e;
    s->seed = seed;
    long nv = e->ph.nvox();
    size_t per_slot = (size_t)s->nbmax * nv * 8;
    if (mem_budget <= 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        mem_budget = (int64_t)std::min<size_t>(fr / 2, (size_t)32 << 30);
    }
    long long fit = (long long)(mem_budget / (int64_t)per_slot);
    if (max_requests <= 0) max_requests = SERVE_MAX;
    s->nslots = (int)std::min<long long>(std::min(fit, (long long)max_requests), SERVE_MAX);
    if (s->nslots < 1)
        return set_err(e, OMC_E_NOMEM, "memory budget holds no request's tallies (" + std::to_string(per_slot) +
                                           " bytes each)");
    if ((rc = s->tallies.alloc(per_slot * s->nslots))) return set_err(e, rc, "server tally allocation failed");
    cudaMemsetAsync(s->tallies.p, 0, per_slot * s->nslots, e->stream);
    if ((rc = s->sdbuf.alloc(sizeof(ServeDev)))) return set_err(e, rc, "server table allocation failed");
    s->sd = s->sdbuf.as<ServeDev>();
    cudaMemsetAsync(s->sd, 0, sizeof(ServeDev), e->stream);
    {
        std::vector<ServeReq> free_req(SERVE_MAX);
        for (auto &q : free_req) q.kind = -1;
        cudaMemcpyAsync(s->sd->req, free_req.data(), sizeof(ServeReq) * SERVE_MAX, cudaMemcpyHostToDevice, e->stream);
    }
    size_t fin = (size_t)nv * (8 * 6 + 4) + NSEG * 8 + 64;
    if ((rc = s->fin.alloc(fin))) return set_err(e, rc, "server finalize allocation failed");
    double *f = s->fin.as<double>();
    s->f_sum = f;
    s->f_sum2 = f + nv;
    s->f_dose = f + 2 * nv;
    s->f_var = f + 3 * nv;
    s->f_vals = f + 4 * nv;
    s->f_vars = f + 5 * nv;
    s->f_rows = (int *)(f + 6 * nv);
    s->f_cnt = s->f_rows + nv;
    s->f_off = s->f_cnt + NSEG;
    s->f_dmax = (unsigned long long *)(((uintptr_t)(s->f_off + NSEG) + 15) / 16 * 16);
    s->f_total = (long long *)(s->f_dmax + 1);
    s->slot_req.assign(s->nslots, -1);
    s->slot_seq.assign(s->nslots, 0);
    {
        // pinned snapshot buffers, their events and the finalisation stream
        size_t per = sizeof(ServeReq) * SERVE_MAX + sizeof(int) * SERVE_MAX + 64 + 8 * sizeof(int);
        if (cudaHostAlloc(&s->snap_host, 2 * per, cudaHostAllocDefault) != cudaSuccess)
            return set_err(e, OMC_E_CUDA, "server snapshot allocation failed");
        for (int k = 0; k < 2; k++) {
            char *b = (char *)s->snap_host + k * per;
            s->snap[k].req = (ServeReq *)b;
            s->snap[k].live = (int *)(b + sizeof(ServeReq) * SERVE_MAX);
            s->snap[k].flags = (unsigned *)(b + sizeof(ServeReq) * SERVE_MAX + sizeof(int) * SERVE_MAX);
            s->snap[k].qc = (int *)(b + sizeof(ServeReq) * SERVE_MAX + sizeof(int) * SERVE_MAX + 64);
            if (cudaEventCreateWithFlags(&s->snap[k].ev, cudaEventDisableTiming) != cudaSuccess)
                return set_err(e, OMC_E_CUDA, "server snapshot event");
        }
        if (cudaStreamCreateWithFlags(&s->fin_stream, cudaStreamNonBlocking) != cudaSuccess)
            return set_err(e, OMC_E_CUDA, "server finalisation stream");
    }
    s->target = std::min<long long>((long long)e->ev->cap / 2, e->ev->inflight);
    if (e->opt.profile) serve_profile_reset(e);
    // reset queue counters and capture two cycles as a graph
    Ctl c0{};
    cudaMemcpyAsync(e->ev->ctl_d, &c0, sizeof(Ctl), cudaMemcpyHostToDevice, e->stream);
    if ((rc = cuda_check(e, cudaStreamSynchronize(e->stream), "server init"))) return rc;
    if ((rc = cuda_check(e, cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal), "capture")))
        return rc;
    serve_launch_cycle(e, 0, s->sd, s->tallies.as<double>(), s->nbmax, s->target);
    serve_launch_cycle(e, 1, s->sd, s->tallies.as<double>(), s->nbmax, s->target);
    if ((rc = cuda_check(e, cudaStreamEndCapture(e->stream, &s->graph), "end capture"))) return rc;
    if ((rc = cuda_check(e, cudaGraphInstantiate(&s->exec, s->graph, 0), "graph instantiate"))) return rc;
    *out = s.release();
    return OMC_OK;
}

int omc_server_destroy(omc_server *s) {
    if (!s) return OMC_OK;
    { std::lock_guard<std::mutex> lk(s->mu); }  // wait for a call in progress
    cudaSetDevice(s->e->device);
    cudaStreamSynchronize(s->e->stream);
    delete s;
    return OMC_OK;
}

int omc_server_completed(omc_server *s, int *ids, int cap, int *n) {
    if (!s || !n || cap < 0 || (cap > 0 && !ids)) return OMC_E_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    int k = std::min<int>(cap, (int)s->completed.size());
    std::copy(s->completed.begin(), s->completed.begin() + k, ids);
    s->completed.erase(s->completed.begin(), s->completed.begin() + k);
    *n = k;
    return OMC_OK;
}

int omc_server_stats(omc_server *s, double *out, int n) {
    if (!s || !out || n < 4) return OMC_E_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    out[0] = (double)s->cycles;
    out[1] = (double)s->drains;
    out[2] = (double)s->launches;
    out[3] = (double)s->finished;
    return OMC_OK;
}

int omc_server_timer(omc_server *s, int stop, double *ms) {
    if (!s) return OMC_E_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    omc_engine *e = s->e;
    cudaSetDevice(e->device);
    if (!s->t_start && (cudaEventCreate(&s->t_start) != cudaSuccess || cudaEventCreate(&s->t_stop) != cudaSuccess))
        return set_err(e, OMC_E_CUDA, "server timer events");
    if (!stop) return cuda_check(e, cudaEventRecord(s->t_start, e->stream), "server timer start");
    int rc = cuda_check(e, cudaEventRecord(s->t_stop, e->stream), "server timer stop");
    if (!rc) rc = cuda_check(e, cudaEventSynchronize(s->t_stop), "server timer stop");
    float m = 0;
    if (!rc) rc = cuda_check(e, cudaEventElapsedTime(&m, s->t_start, s->t_stop), "server timer");
    if (ms) *ms = m;
    return rc;
}

static int submit(omc_server *s, std::unique_ptr<Request> r, uint64_t seed) {
    if (r->nbatch < 2 || r->nbatch > s->nbmax)
        return set_err(s->e, OMC_E_RANGE, "nbatch must be 2.." + std::to_string(s->nbmax));
    if (r->nhist / r->nbatch == 0) r->nhist = r->nbatch;
    r->nper = r->nhist / r->nbatch;
    r->nhist = r->nper * r->nbatch;
    r->id = (int)s->reqs.size();
    r->seed = seed ? mix64(seed) : mix64(s->seed ^ ((uint64_t)(r->id + 1) * 0xD1B54A32D192ED03ull));
    r->t_submit = now_ms();
    int id = r->id;
    s->reqs.push_back(std::move(r));
    s->pending.push_back(id);
    return id;
}

int omc_server_submit_beamlet(omc_server *s, const omc_beamlets *b, int ibixel, int64_t nhist, int nbatch,
                              double rel_threshold, uint64_t seed) {
    if (!s || !b) return OMC_E_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    int rc = check_beamlets(s->e, b);
    if (rc) return rc;
    if (ibixel < 0 || ibixel >= b->nbixels) return set_err(s->e, OMC_E_ARG, "bixel index out of range");
    cudaSetDevice(s->e->device);
    if (!s->plans.count(b)) {
        auto p = std::make_unique<PlanBuf>();
        if ((rc = upload_plan<float>(s->e, b, p->f32, p->s32))) return rc;
        s->plans[b] = std::move(p);
    }
    auto r = std::make_unique<Request>();
    r->kind = 1;
    r->bl = b;
    r->bixel = ibixel;
    r->nhist = nhist;
    r->nbatch = nbatch;
    r->rel = rel_threshold;
    return submit(s, std::move(r), seed);
}

int omc_server_submit_beam(omc_server *s, const omc_beam *b, int64_t nhist, int nbatch, uint64_t seed) {
    if (!s || !b) return OMC_E_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    cudaSetDevice(s->e->device);
    auto r = std::make_unique<Request>();
    r->kind = 0;
    r->beam = *b;
    int n = b->energy.n;
    if (n > 0) {
        if (!b->energy.cdf1 || !b->energy.cdf2) return set_err(s->e, OMC_E_ARG, "spectrum arrays missing");
        std::vector<float> c(b->energy.cdf1, b->energy.cdf1 + n);
        c.insert(c.end(), b->energy.cdf2, b->energy.cdf2 + n);
        int rc = r->cdf.alloc(c.size() * 4);
        if (rc) return set_err(s->e, rc, "alloc");
        cudaMemcpy(r->cdf.p, c.data(), c.size() * 4, cudaMemcpyHostToDevice);
        r->beam.energy.cdf1 = r->beam.energy.cdf2 = nullptr;  // host arrays are not kept
    }
    r->nhist = nhist;
    r->nbatch = nbatch;
    return submit(s, std::move(r), seed);
}

// Queue the snapshot of the request table, live counts, error flags and
// queue counters after the work just queued.
static int take_snapshot(omc_server *s) {
    omc_engine *e = s->e;
    omc_server::Snap &sn = s->snap[s->cur];
    cudaMemcpyAsync(sn.req, s->sd->req, sizeof(ServeReq) * s->nslots, cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(sn.live, s->sd->live, sizeof(int) * s->nslots, cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(sn.flags, &e->ev->ctl_d->flags, sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(sn.qc, e->ev->ctl_d->cnt, 8 * sizeof(int), cudaMemcpyDeviceToHost, e->stream);
    sn.seq = ++s->seq;
    return cuda_check(e, cudaEventRecord(sn.ev, e->stream), "snapshot");
}

// Finish the requests that the snapshot shows complete (all histories
// injected, no particle left) and admit pending ones into the freed slots.
static int process_snapshot(omc_server *s, omc_server::Snap &sn) {
    omc_engine *e = s->e;
    int rc = cuda_check(e, cudaEventSynchronize(sn.ev), "server step");
    if (rc) return rc;
    if (*sn.flags & (ERR_QUEUE | ERR_NAN | ERR_STACK))
        return set_err(e, OMC_E_DEVICE, "device error flags " + std::to_string(*sn.flags) + " in serving");
    // a graph ends with a B -> A cycle: the particles are in queues A
    const long long cap = e->ev->cap;
    const int *qc = sn.qc;
    s->left = std::min<long long>(qc[0] + qc[4], cap) + std::min<long long>(qc[1] + qc[5], cap);
    if (sn.seq <= s->drain_seq) s->left = 0;   // taken before the drain emptied the queues
    s->injected = true;
    std::vector<int> keep;
    bool freed = false;
    for (int slot : s->order) {
        Request &r = *s->reqs[s->slot_req[slot]];
        if (sn.seq <= s->slot_seq[slot]) {   // admitted after this snapshot was taken
            s->injected = false;
            keep.push_back(slot);
            continue;
        }
        const ServeReq &q = sn.req[slot];
        if (q.next < r.nhist) s->injected = false;
        if (q.next >= r.nhist && sn.live[slot] == 0) {
            if ((rc = finalize_request(s, r))) return rc;
            r.state = 2;
            r.t_done = now_ms();
            s->completed.push_back(r.id);
            s->finished++;
            s->slot_req[slot] = -1;
            ServeReq fr{};
            fr.kind = -1;
            cudaMemcpyAsync(&s->sd->req[slot], &fr, sizeof(fr), cudaMemcpyHostToDevice, e->stream);
            freed = true;
        } else {
            keep.push_back(slot);
        }
    }
    sn.seq = 0;
    if (freed) {
        s->order = keep;
        int n = (int)s->order.size();
        if (n) cudaMemcpyAsync(s->sd->order, s->order.data(), n * sizeof(int), cudaMemcpyHostToDevice, e->stream);
        cudaMemcpyAsync(&s->sd->norder, &n, sizeof(int), cudaMemcpyHostToDevice, e->stream);
        if ((rc = cuda_check(e, cudaGetLastError(), "server release"))) return rc;
        if ((rc = admit(s))) return rc;
    }
    return OMC_OK;
}

int omc_server_step(omc_server *s, int cycles, int *active) {
    if (!s) return OMC_E_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    omc_engine *e = s->e;
    cudaSetDevice(e->device);
    int rc = admit(s);
    if (rc) return rc;
    const int prev = s->cur ^ 1;
    if (!s->order.empty()) {
        const long long dthr = drain_threshold(e);
        const int per_cycle = e->d32.d.defer_interact ? 5 : 4;
        if (dthr > 0 && s->injected && s->pending.empty() && s->left > 0 && s->left <= dthr) {
            // the drain's kernel reads the queue sizes on the device; `left`
            // (from the last snapshot, taken before more cycles ran) bounds them
            serve_drain(e, s->sd, s->left, s->tallies.as<double>());
            s->drains++;
            s->launches++;
            s->left = 0;
            s->drain_seq = s->seq;
        } else if (e->opt.profile) {
            // cycles one by one, timed per kernel (the graph's two cycles)
            int graphs = std::max(1, cycles / 2);
            for (int k = 0; k < 2 * graphs; k++)
                if ((rc = serve_profiled_cycle(e, k & 1, s->sd, s->tallies.as<double>(), s->nbmax, s->target)))
                    return rc;
            s->cycles += 2 * graphs;
            s->launches += 2 * graphs * per_cycle;
        } else {
            int graphs = std::max(1, cycles / 2);
            for (int k = 0; k < graphs; k++) cudaGraphLaunch(s->exec, e->stream);
            s->cycles += 2 * graphs;
            s->launches += 2 * graphs * per_cycle;
        }
        if ((rc = take_snapshot(s))) return rc;
        s->cur ^= 1;
    }
    // the previous step's snapshot: ready once the work queued before it is
    if (s->snap[prev].seq > 0 && (rc = process_snapshot(s, s->snap[prev]))) return rc;
    if (s->order.empty() && s->snap[s->cur ^ 1].seq > 0) {
        // nothing running: settle the snapshot just taken too
        if ((rc = process_snapshot(s, s->snap[s->cur ^ 1]))) return rc;
    }
    if (active) *active = (int)(s->order.size() + s->pending.size());
    return OMC_OK;
}

int omc_server_poll(omc_server *s, int id, double *latency_ms) {
    if (!s) return OMC_E_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (id < 0 || id >= (int)s->reqs.size()) return OMC_E_ARG;
    Request &r = *s->reqs[id];
    if (r.state < 2) return OMC_E_NOTREADY;
    if (latency_ms) *latency_ms = r.t_done - r.t_submit;
    return OMC_OK;
}

int omc_server_result_sparse(omc_server *s, int id, int32_t *rows, double *vals, double *var, int64_t cap,
                             int64_t *nnz) {
    if (!s) return OMC_E_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (id < 0 || id >= (int)s->reqs.size() || !nnz) return OMC_E_ARG;
    Request &r = *s->reqs[id];
    if (r.state < 2) return OMC_E_NOTREADY;
    if (r.kind != 1) return set_err(s->e, OMC_E_ARG, "request is not a beamlet");
    *nnz = (int64_t)r.rows.size();
    if ((int64_t)r.rows.size() > cap) return OMC_E_RANGE;
    if (rows) std::copy(r.rows.begin(), r.rows.end(), rows);
    if (vals) std::copy(r.vals.begin(), r.vals.end(), vals);
    if (var) std::copy(r.var.begin(), r.var.end(), var);
    return OMC_OK;
}

int omc_server_result_dense(omc_server *s, int id, double *dose, double *unc) {
    if (!s) return OMC_E_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (id < 0 || id >= (int)s->reqs.size()) return OMC_E_ARG;
    Request &r = *s->reqs[id];
    if (r.state < 2) return OMC_E_NOTREADY;
    if (r.kind != 0) return set_err(s->e, OMC_E_ARG, "request is not a beam");
    if (dose) std::copy(r.dose.begin(), r.dose.end(), dose);
    if (unc) std::copy(r.unc.begin(), r.unc.end(), unc);
    return OMC_OK;
}

int omc_server_release(omc_server *s, int id) {
    if (!s) return OMC_E_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (id < 0 || id >= (int)s->reqs.size()) return OMC_E_ARG;
    Request &r = *s->reqs[id];
    if (r.state < 2) return OMC_E_NOTREADY;
    r.state = 3;
    std::vector<int32_t>().swap(r.rows);
    std::vector<double>().swap(r.vals);
    std::vector<double>().swap(r.var);
    std::vector<double>().swap(r.dose);
    std::vector<double>().swap(r.unc);
    return OMC_OK;
}

// ------------------------------------------------------- matRad D_ij
int omc_run_beamlets(omc_engine *e, const omc_beamlets *b, int64_t nhist, int nbatch, double rel_threshold,
                     uint64_t seed, int mode, int64_t *colptr, int32_t *rows, double *vals, double *var, int64_t cap,
                     int64_t *nnz, double *stats) {
    if (!e || !b || !colptr || !nnz) return OMC_E_ARG;
    int rc = check_beamlets(e, b);
    if (rc) return rc;
    if (nbatch < 2) return set_err(e, OMC_E_ARG, "nbatch must be >= 2");
    cudaSetDevice(e->device);
    int nb = b->nbixels;
    std::vector<std::vector<int32_t>> cr(nb);
    std::vector<std::vector<double>> cv(nb), cvar(nb);
    double t0 = now_ms();
    long long histories = 0;
    double launches = 0;
    if (mode == OMC_EVENT_FP32) {
        if (nbatch > 10) return set_err(e, OMC_E_RANGE, "the event form supports nbatch <= 10");
        omc_server *s = nullptr;
        if ((rc = omc_server_create(e, 0, 0, seed, &s))) return rc;
        std::unique_ptr<omc_server, int (*)(omc_server *)> guard(s, omc_server_destroy);
        std::vector<int> ids(nb);
        for (int i = 0; i < nb; i++) {
            ids[i] = omc_server_submit_beamlet(s, b, i, nhist, nbatch, rel_threshold,
                                               mix64(seed ^ ((uint64_t)(i + 1) * 0x9E3779B97F4A7C15ull)));
            if (ids[i] < 0) return ids[i];
        }
        int active = nb;
        long long guard_cycles = 0;
        while (active > 0) {
            if ((rc = omc_server_step(s, 8, &active))) return rc;
            if (++guard_cycles > 10000000) return set_err(e, OMC_E_DEVICE, "serving did not drain");
        }
        for (int i = 0; i < nb; i++) {
            Request &r = *s->reqs[ids[i]];
            cr[i] = std::move(r.rows);
            cv[i] = std::move(r.vals);
            cvar[i] = std::move(r.var);
            histories += r.nhist;
        }
        launches = (double)s->cycles * (e->d32.d.defer_interact ? 5 : 4) + (double)s->drains;
    } else if (mode == OMC_PLAIN_FP64) {
        PlanBuf pb;
        if ((rc = upload_plan<double>(e, b, pb.f64, pb.s64))) return rc;
        long nv = e->ph.nvox();
        DBuf work, fin;
        if ((rc = work.alloc(nv * 8))) return set_err(e, rc, "alloc");
        size_t finb = (size_t)nv * (8 * 6 + 4) + NSEG * 8 + 64;
        if ((rc = fin.alloc(finb))) return set_err(e, rc, "alloc");
        cudaMemsetAsync(work.p, 0, nv * 8, e->stream);
        double *f = fin.as<double>();
        double *sum = f, *sum2 = f + nv, *dose = f + 2 * nv, *vv = f + 3 * nv, *fvals = f + 4 * nv, *fvars = f + 5 * nv;
        int *frows = (int *)(f + 6 * nv), *cnt = frows + nv, *off = cnt + NSEG;
        unsigned long long *dmax = (unsigned long long *)(((uintptr_t)(off + NSEG) + 15) / 16 * 16);
        long long *total = (long long *)(dmax + 1);
        if (nhist / nbatch == 0) nhist = nbatch;
        long nper = (long)(nhist / nbatch);
        int block = e->opt.block > 0 ? e->opt.block : 128;
        // ompMC keeps accumulating sum2 over beamlets (omc_matrad.c:1702 resets
        // only accum_endep): reproduced with ref_compat
        cudaMemsetAsync(sum2, 0, nv * 8, e->stream);
        for (int i = 0; i < nb; i++) {
            cudaMemsetAsync(sum, 0, nv * 8, e->stream);
            if (!e->opt.ref_compat) cudaMemsetAsync(sum2, 0, nv * 8, e->stream);
            for (int bt = 0; bt < nbatch; bt++) {
                if ((rc = plain_beamlet_batch(e, pb.s64, i, work.as<double>(), seed, (long)bt * nper, nper, block)))
                    return rc;
                if ((rc = fold(e, work.as<double>(), sum, sum2, nv, 1.0 / (double)nper))) return rc;
            }
            if ((rc = finalize_matrad(e, sum, sum2, nbatch, dose, vv))) return rc;
            cudaMemsetAsync(dmax, 0, 8, e->stream);
            int g = std::max(1, std::min((int)((nv + 255) / 256), e->sm_count * 4));
            k_dmax<<<g, 256, 0, e->stream>>>(dose, nv, dmax);
            long seglen = (nv + NSEG - 1) / NSEG;
            k_seg_count<<<NSEG, 256, 0, e->stream>>>(dose, nv, seglen, dmax, rel_threshold, cnt);
            k_seg_scan<<<1, NSEG, 0, e->stream>>>(cnt, off, total);
            k_seg_write<<<NSEG, 256, 0, e->stream>>>(dose, vv, nv, seglen, dmax, rel_threshold, off, frows, fvals,
                                                      fvars, nv);
            long long n = 0;
            cudaMemcpyAsync(&n, total, 8, cudaMemcpyDeviceToHost, e->stream);
            if ((rc = cuda_check(e, cudaStreamSynchronize(e->stream), "plain beamlet"))) return rc;
            cr[i].resize(n);
            cv[i].resize(n);
            cvar[i].resize(n);
            if (n) {
                cudaMemcpy(cr[i].data(), frows, n * 4, cudaMemcpyDeviceToHost);
                cudaMemcpy(cv[i].data(), fvals, n * 8, cudaMemcpyDeviceToHost);
                cudaMemcpy(cvar[i].data(), fvars, n * 8, cudaMemcpyDeviceToHost);
            }
            histories += (long long)nper * nbatch;
            launches += 2.0 * nbatch + 5;
        }
        unsigned flags = 0;
        cudaMemcpy(&flags, e->errword.p, sizeof(unsigned), cudaMemcpyDeviceToHost);
        if (flags & (ERR_STACK | ERR_NAN)) return set_err(e, OMC_E_DEVICE, "device error flags in plain beamlets");
    } else {
        return set_err(e, OMC_E_ARG, "unknown mode");
    }
    int64_t total = 0;
    colptr[0] = 0;
    for (int i = 0; i < nb; i++) {
        total += (int64_t)cr[i].size();
        colptr[i + 1] = total;
    }
    *nnz = total;
    if (stats) {
        stats[0] = (double)histories;
        stats[1] = (now_ms() - t0) * 1e-3;
        stats[2] = launches;
        stats[3] = stats[4] = stats[5] = 0;
    }
    if (total > cap) return set_err(e, OMC_E_RANGE, "sparse capacity " + std::to_string(cap) + " < " + std::to_string(total));
    int64_t o = 0;
    for (int i = 0; i < nb; i++) {
        if (rows) std::copy(cr[i].begin(), cr[i].end(), rows + o);
        if (vals) std::copy(cv[i].begin(), cv[i].end(), vals + o);
        if (var) std::copy(cvar[i].begin(), cvar[i].end(), var + o);
        o += (int64_t)cr[i].size();
    }
    return OMC_OK;
}

}  // extern "C"
