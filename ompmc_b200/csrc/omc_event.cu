// Event-based FP32 transport: structure-of-arrays particle queues, one
// transport event (one call of ompMC's photon() or electron(), until the next
// interaction or death) per thread per launch, outputs appended with
// warp-aggregated atomics, FP64 tallies per batch slot.
//
// A transport cycle is five launches on one stream:
//   k_plan      how many new histories fit (in-flight target - occupancy)
//   k_source    primaries of those histories into the input queues
//   k_photon    one photon event per queued photon
//   k_electron  one electron event per queued e-/e+
//   k_reset     input queues consumed
// Queues are double-buffered (A -> B, then B -> A), so two cycles form an
// idempotent CUDA graph that the host replays until every history is done.
// Each particle carries its own Philox stream (key, block counter), so the
// result does not depend on scheduling.
#include <algorithm>
#include <cstdio>

#include "omc_event.h"
#include "omc_rng.cuh"
#include "omc_source.cuh"

namespace omc {

constexpr int EV_BUDGET = 200000;  // transport steps one event may take
constexpr int EV_MAXOUT = 3;       // particles an event may emit

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

struct EvEnv {
    Philox<float> rng;
    double *tally;
    int pend_ir;
    double pend_e;
    Part<float> out[EV_MAXOUT];
    int nout;
    unsigned flags;
    int work;
    int ncross, ndep, natom;
    __device__ float uni() { return rng.uni(); }
    // Consecutive deposits into one voxel are summed before the atomic.
    __device__ void deposit(int ir, float e) {
        ndep++;
        if (ir != pend_ir) {
            flush();
            pend_ir = ir;
        }
        pend_e += (double)e;
    }
    __device__ void flush() {
        if (pend_ir > 0 && pend_e != 0.0) {
            atomicAdd(&tally[pend_ir - 1], pend_e);
            natom++;
        }
        pend_e = 0.0;
        pend_ir = -1;
    }
    __device__ void cross() { ncross++; }
    int tsteps;
    __device__ int tstep_budget() const { return tsteps; }
    __device__ bool push(const Part<float> &q) {
        if (nout >= EV_MAXOUT) {
            flags |= ERR_STACK;
            return false;
        }
        out[nout++] = q;
        return true;
    }
    __device__ void err(unsigned f) { flags |= f; }
    __device__ bool tick() { return ++work < EV_BUDGET; }
};

struct SrcEnv {
    Philox<float> rng;
    __device__ float uni() { return rng.uni(); }
};

__device__ __forceinline__ void qload(const Queue &q, int i, Part<float> &p, int &tag, uint32_t &k0, uint32_t &k1,
                                      uint32_t &ctr) {
    p.x = q.x[i]; p.y = q.y[i]; p.z = q.z[i];
    p.u = q.u[i]; p.v = q.v[i]; p.w = q.w[i];
    p.e = q.e[i]; p.wt = q.wt[i];
    p.ir = q.ir[i];
    tag = q.tag[i];
    p.iq = (tag & 3) - 1;
    k0 = q.k0[i]; k1 = q.k1[i]; ctr = q.ctr[i];
}

__device__ __forceinline__ void qstore(const Queue &q, int i, const Part<float> &p, int slot, uint32_t k0, uint32_t k1,
                                       uint32_t ctr) {
    q.x[i] = p.x; q.y[i] = p.y; q.z[i] = p.z;
    q.u[i] = p.u; q.v[i] = p.v; q.w[i] = p.w;
    q.e[i] = p.e; q.wt[i] = p.wt;
    q.ir[i] = p.ir;
    q.tag[i] = (p.iq + 1) | (slot << 2);
    q.k0[i] = k0; q.k1[i] = k1; q.ctr[i] = ctr;
}

// Slot of a warp-aggregated append to `q` for the lanes with `want`;
// -1 for the others (or on overflow, flagged).
__device__ __forceinline__ int warp_append(const Queue &q, bool want, unsigned active, unsigned &flags) {
    unsigned m = __ballot_sync(active, want);
    if (!m) return -1;
    int lane = threadIdx.x & 31;
    int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(q.count, __popc(m));
    base = __shfl_sync(active, base, leader);
    if (!want) return -1;
    int idx = base + __popc(m & lanemask_lt());
    if (idx >= q.cap) {
        flags |= ERR_QUEUE;
        return -1;
    }
    return idx;
}

__device__ __forceinline__ void renorm(Part<float> &p) {
    float n2 = p.u * p.u + p.v * p.v + p.w * p.w;
    if (n2 > 0.f && fabsf(n2 - 1.f) > 1e-6f) {
        float r = rsqrtf(n2);
        p.u *= r; p.v *= r; p.w *= r;
    }
}

// Route the event's surviving particle and its secondaries to the output
// queues.  Secondaries get fresh streams derived from the parent's key and
// block counter, which is unique per event.  Returns the particles queued.
__device__ __forceinline__ int emit(const Queue &outP, const Queue &outE, unsigned active, bool alive,
                                    Part<float> &p, EvEnv &g, int slot, uint32_t k0, uint32_t k1) {
    uint64_t pkey = ((uint64_t)k1 << 32) | k0;
    uint32_t pctr = g.rng.ctr;
    int queued = 0;
#pragma unroll
    for (int k = 0; k < 1 + EV_MAXOUT; k++) {
        bool has;
        Part<float> q;
        if (k == 0) {
            has = alive;
            q = p;
        } else {
            has = k - 1 < g.nout;
            q = g.out[k - 1 < EV_MAXOUT ? k - 1 : 0];
        }
        if (__ballot_sync(active, has) == 0) continue;
        if (has) renorm(q);
        if (has && !(q.e == q.e && q.x == q.x && q.u == q.u)) {
            g.flags |= ERR_NAN;
            has = false;
        }
        bool isph = has && q.iq == 0;
        bool isel = has && q.iq != 0;
        int ip = warp_append(outP, isph, active, g.flags);
        int ie = warp_append(outE, isel, active, g.flags);
        uint32_t a0 = k0, a1 = k1, ac = pctr;
        if (k > 0) {
            uint64_t ck = mix64(pkey * 0x9E3779B97F4A7C15ull + ((uint64_t)pctr << 3) + (uint64_t)k);
            a0 = (uint32_t)ck;
            a1 = (uint32_t)(ck >> 32);
            ac = 0;
        }
        if (ip >= 0) qstore(outP, ip, q, slot, a0, a1, ac);
        if (ie >= 0) qstore(outE, ie, q, slot, a0, a1, ac);
        queued += (ip >= 0) + (ie >= 0);
    }
    return queued;
}

__device__ __forceinline__ void report_flags(Ctl *ctl, unsigned flags, unsigned active) {
    unsigned f = __reduce_or_sync(active, flags);
    if (f && (threadIdx.x & 31) == __ffs(active) - 1) atomicOr(&ctl->flags, f);
}

__device__ __forceinline__ void report_count(unsigned long long *dst, unsigned v, unsigned active) {
    unsigned t = __reduce_add_sync(active, v);
    if (t && (threadIdx.x & 31) == __ffs(active) - 1) atomicAdd(dst, (unsigned long long)t);
}

// Live-particle count of a serving request: +delta for the request whose
// tally slots start at req*nbmax, aggregated over the lanes of the warp that
// hold particles of the same request.
__device__ __forceinline__ void add_live(int *live, int nbmax, int slot, int delta, unsigned active) {
    int req = slot / nbmax;
    unsigned grp = __match_any_sync(active, req);
    int tot = __reduce_add_sync(grp, delta);
    if (tot != 0 && (threadIdx.x & 31) == __ffs(grp) - 1) atomicAdd(&live[req], tot);
}

template <bool PHOTON>
__device__ __forceinline__ void transport_events(const DevData<float> &D, const Queue &in, const Queue &outP,
                                                 const Queue &outE, double *tallies, long nvox, Ctl *ctl,
                                                 uint32_t seedw, int tsteps, int *live, int nbmax) {
    int n = min(*in.count, in.cap);
    unsigned flags = 0;
    unsigned c_ev = 0, c_steps = 0, c_cross = 0, c_dep = 0, c_atom = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        unsigned active = __activemask();
        Part<float> p;
        int tag;
        uint32_t k0, k1, ctr;
        qload(in, i, p, tag, k0, k1, ctr);
        int slot = tag >> 2;
        EvEnv g;
        g.rng.init(((uint64_t)k1 << 32) | k0, seedw, ctr);
        g.tally = tallies + (long)slot * nvox;
        g.pend_ir = -1;
        g.pend_e = 0.0;
        g.nout = 0;
        g.flags = 0;
        g.work = 0;
        g.tsteps = tsteps;
        g.ncross = g.ndep = g.natom = 0;
        bool alive;
        if (PHOTON) alive = photon_step(D, g, p);
        else alive = electron_step(D, g, p) == E_ALIVE;
        g.flush();
        int emitted = emit(outP, outE, active, alive, p, g, slot, k0, k1);
        if (live) add_live(live, nbmax, slot, emitted - 1, active);
        flags |= g.flags;
        c_ev++;
        c_steps += g.work;
        c_cross += g.ncross;
        c_dep += g.ndep;
        c_atom += g.natom;
    }
    unsigned active = __activemask();
    report_flags(ctl, flags, active);
    const int k = PHOTON ? 0 : 1;
    report_count(&ctl->st_events[k], c_ev, active);
    report_count(&ctl->st_steps[k], c_steps, active);
    report_count(&ctl->st_cross[k], c_cross, active);
    report_count(&ctl->st_dep[k], c_dep, active);
    report_count(&ctl->st_atom[k], c_atom, active);
}

// One photon event per queued photon.  `live` (may be null) receives the
// change of each serving request's live-particle count.
__global__ void __launch_bounds__(256) k_photon_step(DevData<float> D, Queue in, Queue outP, Queue outE,
                                                     double *tallies, long nvox, Ctl *ctl, uint32_t seedw,
                                                     int *live, int nbmax) {
    transport_events<true>(D, in, outP, outE, tallies, nvox, ctl, seedw, 1 << 30, live, nbmax);
}

// One bounded electron/positron event per queued charged particle: at most
// `tsteps` iterations of electron()'s tstep loop, then the particle is
// re-queued, so every lane of a warp does a similar amount of work.
__global__ void __launch_bounds__(256) k_electron_step(DevData<float> D, Queue in, Queue outP, Queue outE,
                                                       double *tallies, long nvox, Ctl *ctl, uint32_t seedw,
                                                       int tsteps, int *live, int nbmax) {
    transport_events<false>(D, in, outP, outE, tallies, nvox, ctl, seedw, tsteps, live, nbmax);
}

__global__ void k_source(DevData<float> D, BeamSrc<float> S, Queue qP, Queue qE, Ctl *ctl, long long nper,
                         uint64_t seed, uint32_t seedw) {
    int n = ctl->inject;
    long long base = ctl->hist_base;
    double es = 0;
    unsigned flags = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        unsigned active = __activemask();
        long long h = base + i;
        SrcEnv g;
        uint64_t key = mix64(seed ^ (uint64_t)h * 0x9E3779B97F4A7C15ull);
        g.rng.init(key, seedw);
        float ein;
        Part<float> p = beam_primary(D, S, g, ein);
        es += ein;
        int slot = (int)(h / nper);
        int ip = warp_append(qP, p.iq == 0, active, flags);
        int ie = warp_append(qE, p.iq != 0, active, flags);
        if (ip >= 0) qstore(qP, ip, p, slot, (uint32_t)key, (uint32_t)(key >> 32), g.rng.ctr);
        if (ie >= 0) qstore(qE, ie, p, slot, (uint32_t)key, (uint32_t)(key >> 32), g.rng.ctr);
    }
    for (int o = 16; o > 0; o >>= 1) es += __shfl_down_sync(0xffffffffu, es, o);
    if ((threadIdx.x & 31) == 0 && es != 0.0) atomicAdd(&ctl->src_energy, es);
    unsigned active = __activemask();
    report_flags(ctl, flags, active);
}

// Histories to inject this cycle: keep `target` particles in flight.
__global__ void k_plan(Ctl *ctl, int iph, int iel, long long target, int cap) {
    long long occ = (long long)min(ctl->cnt[iph], cap) + min(ctl->cnt[iel], cap);
    long long rem = ctl->hist_total - ctl->hist_next;
    long long inj = target - occ;
    if (inj < 0) inj = 0;
    if (inj > rem) inj = rem;
    long long room = (long long)cap - ctl->cnt[iph];
    if (inj > room) inj = room > 0 ? room : 0;
    ctl->inject = (int)inj;
    ctl->hist_base = ctl->hist_next;
    ctl->hist_next += inj;
}

__global__ void k_reset(Ctl *ctl, int iph, int iel) {
    ctl->cnt[iph] = 0;
    ctl->cnt[iel] = 0;
}

// ------------------------------------------------------------------ host
static int alloc_queue(omc_engine *e, DBuf &b, Queue &q, int cap, int *count) {
    size_t per = (size_t)cap * 4;
    int rc = b.alloc(per * 13);
    if (rc) return set_err(e, rc, "event queue allocation failed");
    char *p = (char *)b.p;
    float **f[8] = {&q.x, &q.y, &q.z, &q.u, &q.v, &q.w, &q.e, &q.wt};
    for (int i = 0; i < 8; i++) *f[i] = (float *)(p + per * i);
    q.ir = (int *)(p + per * 8);
    q.tag = (int *)(p + per * 9);
    q.k0 = (uint32_t *)(p + per * 10);
    q.k1 = (uint32_t *)(p + per * 11);
    q.ctr = (uint32_t *)(p + per * 12);
    q.count = count;
    q.cap = cap;
    return OMC_OK;
}

int event_prepare(omc_engine *e) {
    if (e->ev && e->ev->ready) return OMC_OK;
    if (!e->ev) e->ev = new EventState();
    EventState &S = *e->ev;
    long cap = e->opt.queue_capacity > 0 ? e->opt.queue_capacity : (1L << 22);
    S.cap = (int)std::min(cap, (long)(1L << 30));
    S.block = e->opt.block > 0 ? e->opt.block : 256;
    S.grid = e->sm_count * (2048 / S.block);
    // 2 measured best on the slab workload (sweep of 1..16 on a B200)
    S.tsteps = e->opt.electron_tsteps > 0 ? e->opt.electron_tsteps : 2;
    S.inflight = e->opt.inflight > 0 ? e->opt.inflight : (1LL << 20);
    int rc = S.ctl.alloc(sizeof(Ctl));
    if (rc) return set_err(e, rc, "control block allocation failed");
    S.ctl_d = S.ctl.as<Ctl>();
    for (int i = 0; i < 4; i++)
        if ((rc = alloc_queue(e, S.buf[i], S.q[i], S.cap, &S.ctl_d->cnt[i]))) return rc;
    S.ready = true;
    return OMC_OK;
}

void event_release(omc_engine *e) {
    delete e->ev;
    e->ev = nullptr;
}

// One transport cycle with input buffers `in` (0 = A, 1 = B).  With `ev`
// (profiling) an event is recorded before each launch and after the last.
static void launch_cycle(omc_engine *e, int in, const BeamSrc<float> &src, double *tallies, long nper, uint64_t seed,
                         long long target, cudaEvent_t *ev = nullptr) {
    EventState &S = *e->ev;
    int iph = in == 0 ? 0 : 2, iel = iph + 1;
    int oph = in == 0 ? 2 : 0, oel = oph + 1;
    uint32_t seedw = (uint32_t)(seed >> 32);
    long nvox = e->ph.nvox();
    if (ev) cudaEventRecord(ev[0], e->stream);
    k_plan<<<1, 1, 0, e->stream>>>(S.ctl_d, iph, iel, target, S.cap);
    if (ev) cudaEventRecord(ev[1], e->stream);
    k_source<<<S.grid, S.block, 0, e->stream>>>(e->d32.d, src, S.q[iph], S.q[iel], S.ctl_d, nper, seed, seedw);
    if (ev) cudaEventRecord(ev[2], e->stream);
    k_photon_step<<<S.grid, S.block, 0, e->stream>>>(e->d32.d, S.q[iph], S.q[oph], S.q[oel], tallies, nvox,
                                                          S.ctl_d, seedw, nullptr, 1);
    if (ev) cudaEventRecord(ev[3], e->stream);
    k_electron_step<<<S.grid, S.block, 0, e->stream>>>(e->d32.d, S.q[iel], S.q[oph], S.q[oel], tallies, nvox,
                                                           S.ctl_d, seedw, S.tsteps, nullptr, 1);
    if (ev) cudaEventRecord(ev[4], e->stream);
    k_reset<<<1, 1, 0, e->stream>>>(S.ctl_d, iph, iel);
    if (ev) cudaEventRecord(ev[5], e->stream);
}

// Profiled transport: cycles launched one by one with events around each
// kernel; per-kernel device time accumulated into S.prof.
static int run_profiled(omc_engine *e, const BeamSrc<float> &src, double *tallies, long nper, uint64_t seed,
                        long long target, Ctl &h, long &cycles) {
    EventState &S = *e->ev;
    for (auto &p : S.prof) p = KernelProfile();
    S.trace.clear();
    cudaEvent_t ev[6];
    for (auto &x : ev) cudaEventCreate(&x);
    int rc = OMC_OK;
    cycles = 0;
    int cnt_in[2] = {0, 0};   // queue sizes the cycle starts with (before injection)
    for (;;) {
        int in = (int)(cycles & 1);
        launch_cycle(e, in, src, tallies, nper, seed, target, ev);
        cycles++;
        if ((rc = cuda_check(e, cudaEventSynchronize(ev[5]), "profiled cycle"))) break;
        float t[5];
        for (int k = 0; k < 5; k++) cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]);
        Ctl c;
        cudaMemcpy(&c, S.ctl_d, sizeof(Ctl), cudaMemcpyDeviceToHost);
        int oph = in == 0 ? 2 : 0;
        double row[6] = {(double)c.inject, (double)cnt_in[0] + c.inject, (double)cnt_in[1], t[1], t[2], t[3]};
        S.trace.insert(S.trace.end(), row, row + 6);
        cnt_in[0] = std::min(c.cnt[oph], S.cap);
        cnt_in[1] = std::min(c.cnt[oph + 1], S.cap);
        S.prof[3].seconds += (t[0] + t[4]) * 1e-3;
        S.prof[3].launches += 2;
        S.prof[0].seconds += t[1] * 1e-3;
        S.prof[0].launches += 1;
        S.prof[1].seconds += t[2] * 1e-3;
        S.prof[1].launches += 1;
        S.prof[2].seconds += t[3] * 1e-3;
        S.prof[2].launches += 1;
        if ((cycles & 1) == 0) {
            cudaMemcpy(&h, S.ctl_d, sizeof(Ctl), cudaMemcpyDeviceToHost);
            if (h.hist_next >= h.hist_total && h.cnt[0] == 0 && h.cnt[1] == 0) break;
            if (h.flags & ERR_QUEUE) break;
        }
        if (cycles > 200000) {
            rc = set_err(e, OMC_E_DEVICE, "event transport did not drain");
            break;
        }
    }
    for (auto &x : ev) cudaEventDestroy(x);
    return rc;
}

int event_run_beam(omc_engine *e, const omc_beam *b, long nper, int nbatch, uint64_t seed, double *sum, double *sum2,
                   double *src_energy, KernelStats &ks) {
    int rc = event_prepare(e);
    if (rc) return rc;
    EventState &S = *e->ev;
    long nvox = e->ph.nvox();
    DBuf tal, cdf;
    if ((rc = tal.alloc((size_t)nbatch * nvox * 8))) return set_err(e, rc, "batch tallies allocation failed");
    cudaMemsetAsync(tal.p, 0, (size_t)nbatch * nvox * 8, e->stream);
    int ncdf = b->energy.n;
    BeamSrc<float> src = beam_setup<float>(e, b);
    if (ncdf > 0) {
        std::vector<float> c(b->energy.cdf1, b->energy.cdf1 + ncdf);
        c.insert(c.end(), b->energy.cdf2, b->energy.cdf2 + ncdf);
        if ((rc = cdf.alloc(c.size() * 4))) return set_err(e, rc, "alloc");
        cudaMemcpyAsync(cdf.p, c.data(), c.size() * 4, cudaMemcpyHostToDevice, e->stream);
        src.cdf1 = cdf.as<float>();
        src.cdf2 = cdf.as<float>() + ncdf;
    }
    Ctl c0{};
    c0.hist_total = (long long)nper * nbatch;
    cudaMemcpyAsync(S.ctl_d, &c0, sizeof(Ctl), cudaMemcpyHostToDevice, e->stream);
    long long target = std::min<long long>((long long)S.cap / 2, S.inflight);

    if (e->opt.profile) {
        Ctl h{};
        long cycles = 0;
        cudaEvent_t t0, t1;
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, e->stream);
        rc = run_profiled(e, src, tal.as<double>(), nper, seed, target, h, cycles);
        for (int ib = 0; ib < nbatch && rc == OMC_OK; ib++)
            rc = fold(e, tal.as<double>() + (size_t)ib * nvox, sum, sum2, nvox, 1.0);
        cudaEventRecord(t1, e->stream);
        cudaEventSynchronize(t1);
        float ms = 0;
        cudaEventElapsedTime(&ms, t0, t1);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        ks.seconds = ms * 1e-3;
        ks.launches = cycles * 5 + nbatch;
        ks.flags |= h.flags;
        for (int k = 0; k < 2; k++) {
            KernelProfile &P = S.prof[1 + k];
            P.particles = (double)h.st_events[k];
            P.steps = (double)h.st_steps[k];
            P.cross = (double)h.st_cross[k];
            P.dep = (double)h.st_dep[k];
            P.atom = (double)h.st_atom[k];
        }
        S.prof[0].particles = (double)h.hist_total;
        if (rc) return rc;
        cudaMemcpyAsync(src_energy, &S.ctl_d->src_energy, 8, cudaMemcpyDeviceToDevice, e->stream);
        return OMC_OK;
    }

    // capture two cycles (A -> B, B -> A) as one graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if ((rc = cuda_check(e, cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal), "capture"))) return rc;
    launch_cycle(e, 0, src, tal.as<double>(), nper, seed, target);
    launch_cycle(e, 1, src, tal.as<double>(), nper, seed, target);
    if ((rc = cuda_check(e, cudaStreamEndCapture(e->stream, &graph), "end capture"))) return rc;
    if ((rc = cuda_check(e, cudaGraphInstantiate(&exec, graph, 0), "graph instantiate"))) {
        cudaGraphDestroy(graph);
        return rc;
    }
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, e->stream);
    Ctl h{};
    long graphs = 0;
    int per_check = 4;
    for (;;) {
        for (int k = 0; k < per_check; k++) cudaGraphLaunch(exec, e->stream);
        graphs += per_check;
        cudaMemcpyAsync(&h, S.ctl_d, sizeof(Ctl), cudaMemcpyDeviceToHost, e->stream);
        if ((rc = cuda_check(e, cudaStreamSynchronize(e->stream), "event transport"))) break;
        if (h.hist_next >= h.hist_total && h.cnt[0] == 0 && h.cnt[1] == 0 && h.cnt[2] == 0 && h.cnt[3] == 0) break;
        if (h.flags & ERR_QUEUE) break;
        // every cycle advances each queued particle by one event, so a run
        // needs (histories / injection rate) + (longest history) cycles
        if (graphs > 50000 + h.hist_total / 1000) {
            rc = set_err(e, OMC_E_DEVICE, "event transport did not drain");
            break;
        }
        per_check = std::min(per_check * 2, 64);
    }
    // fold the batch tallies into the sums (accumEndep per batch)
    for (int ib = 0; ib < nbatch && rc == OMC_OK; ib++)
        rc = fold(e, tal.as<double>() + (size_t)ib * nvox, sum, sum2, nvox, 1.0);
    cudaEventRecord(t1, e->stream);
    cudaEventSynchronize(t1);
    float ms = 0;
    cudaEventElapsedTime(&ms, t0, t1);
    ks.seconds = ms * 1e-3;
    ks.launches = graphs * 10 + nbatch;
    ks.flags |= h.flags;
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc) return rc;
    // source energy
    cudaMemcpyAsync(src_energy, &S.ctl_d->src_energy, 8, cudaMemcpyDeviceToDevice, e->stream);
    return OMC_OK;
}

// ============================================================== serving
// Histories to inject this cycle across the admitted requests, first come
// first served, keeping `target` particles in flight.
__global__ void k_serve_plan(ServeDev *sd, Ctl *ctl, int iph, int iel, long long target, int cap) {
    long long occ = (long long)min(ctl->cnt[iph], cap) + min(ctl->cnt[iel], cap);
    long long room = target - occ;
    long long qroom = (long long)cap - max(ctl->cnt[iph], ctl->cnt[iel]);
    if (room > qroom) room = qroom;
    int np = 0;
    long long cum = 0;
    for (int k = 0; k < sd->norder && room - cum > 0; k++) {
        int s = sd->order[k];
        ServeReq &r = sd->req[s];
        if (r.kind < 0) continue;
        long long rem = r.nhist - r.next;
        if (rem <= 0) continue;
        long long take = rem < room - cum ? rem : room - cum;
        sd->plan_slot[np] = s;
        sd->plan_first[np] = r.next;
        sd->plan_cum[np] = (int)cum;
        cum += take;
        r.next += take;
        np++;
    }
    sd->plan_cum[np] = (int)cum;
    sd->nplan = np;
    sd->inject_total = (int)cum;
}

// Primaries of the planned histories; each history's stream key is derived
// from its request's seed and its index within the request.
__global__ void k_serve_source(DevData<float> D, ServeDev *sd, Queue qP, Queue qE, Ctl *ctl, int nbmax,
                               uint32_t seedw) {
    int n = sd->inject_total, np = sd->nplan;
    unsigned flags = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        unsigned active = __activemask();
        int lo = 0, hi = np - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (sd->plan_cum[mid] <= i) lo = mid;
            else hi = mid - 1;
        }
        int s = sd->plan_slot[lo];
        const ServeReq &r = sd->req[s];
        long long local = sd->plan_first[lo] + (i - sd->plan_cum[lo]);
        uint64_t key = mix64(r.seed ^ (uint64_t)local * 0x9E3779B97F4A7C15ull);
        SrcEnv g;
        g.rng.init(key, seedw);
        float ein;
        Part<float> p = r.kind == 0 ? beam_primary(D, sd->beam[s], g, ein) : beamlet_primary(D, sd->bl[s], r.bixel, g, ein);
        int slot = s * nbmax + (int)(local / r.nper);
        int ip = warp_append(qP, p.iq == 0, active, flags);
        int ie = warp_append(qE, p.iq != 0, active, flags);
        if (ip >= 0) qstore(qP, ip, p, slot, (uint32_t)key, (uint32_t)(key >> 32), g.rng.ctr);
        if (ie >= 0) qstore(qE, ie, p, slot, (uint32_t)key, (uint32_t)(key >> 32), g.rng.ctr);
        add_live(sd->live, nbmax, slot, (ip >= 0) + (ie >= 0), active);
    }
    unsigned active = __activemask();
    report_flags(ctl, flags, active);
}

void serve_launch_cycle(omc_engine *e, int in, ServeDev *sd, double *tallies, int nbmax, long long target) {
    EventState &S = *e->ev;
    int iph = in == 0 ? 0 : 2, iel = iph + 1;
    int oph = in == 0 ? 2 : 0, oel = oph + 1;
    uint32_t seedw = 0x5e7e5eedu;
    long nvox = e->ph.nvox();
    k_serve_plan<<<1, 1, 0, e->stream>>>(sd, S.ctl_d, iph, iel, target, S.cap);
    k_serve_source<<<S.grid, S.block, 0, e->stream>>>(e->d32.d, sd, S.q[iph], S.q[iel], S.ctl_d, nbmax, seedw);
    k_photon_step<<<S.grid, S.block, 0, e->stream>>>(e->d32.d, S.q[iph], S.q[oph], S.q[oel], tallies, nvox, S.ctl_d,
                                                      seedw, sd->live, nbmax);
    k_electron_step<<<S.grid, S.block, 0, e->stream>>>(e->d32.d, S.q[iel], S.q[oph], S.q[oel], tallies, nvox,
                                                        S.ctl_d, seedw, S.tsteps, sd->live, nbmax);
    k_reset<<<1, 1, 0, e->stream>>>(S.ctl_d, iph, iel);
}

}  // namespace omc
