// Event-based FP32 transport: structure-of-arrays particle queues, one
// transport event per queued particle per launch, outputs appended with
// warp-aggregated atomics, FP64 tallies per batch slot.
//
// A transport cycle is five launches on one stream:
//   k_plan      how many new histories fit (in-flight target - occupancy),
//               the electron budget of this cycle, output queues emptied
//   k_source    primaries of those histories into the input queues
//   k_photon    one photon event per queued photon
//   k_electron  one electron event per queued e-/e+; electrons that reach a
//               discrete interaction are queued for
//   k_electron_interact  which samples those interactions (a kernel of its
//               own keeps the samplers' code out of the transport kernel's
//               instruction cache: 8 % faster on slab64)
// Queues are double-buffered (A -> B, then B -> A), so two cycles form an
// idempotent CUDA graph that the host replays until every history is
// injected and few particles are left; k_drain then runs those to the end.
//
// An event transports its particle until the next interaction, death or,
// for electrons, the end of the cycle's budget of tstep-loop iterations.
// The budget is small while the queues fill the GPU (lanes of a warp then do
// similar work) and grows as they drain, so the drain tail takes few
// cycles.  Each particle carries its own Philox stream (key, position) and
// secondaries get keys from the parent's key and stream position at their
// creation, so a particle's trajectory does not depend on where events are
// cut nor on scheduling: any budget gives the same result up to the
// summation order of the FP64 tallies.
#include <algorithm>
#include <cstdio>

#include "omc_event.h"


#include "omc_rng.cuh"
#include "omc_source.cuh"

namespace omc {

constexpr int EV_BUDGET = 200000;  // transport steps one event may take
constexpr int EV_MAXOUT = 1;       // secondaries an event emits: every interaction sampler pushes one
constexpr int EV_MAXOUT_SPLIT = 2; // products of a split photon's sub-photon (pair: two)
constexpr int EV_MAX_BLOCK = 256;  // launch bound of the transport kernels
// Resident 256-thread blocks per SM the electron kernel is compiled for:
// four (64 registers) in FP32, two (128 registers) in FP64.  Measured on the
// served beamlet load and the slab beam with the step's state in
// registers: 3 blocks (80 registers) 50.6 and 70.3 M hist/s, 4 blocks 52.6
// and 71.8, 5 blocks (48 registers) 52.1 and 70.3.
template <typename R>
constexpr int electron_minb() {
    return sizeof(R) == 4 ? 4 : 2;
}

template <typename R>
using TransportKernelT = void (*)(DevData<R>, QueueT<R>, QueueT<R>, QueueT<R>, double *, long, Ctl *, uint32_t,
                                  ServeDev *, int, QueueT<R>);
using TransportKernel = TransportKernelT<float>;

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <int MAXOUT, typename R = float>
struct EvEnv {
    Philox<R> rng;
    double *tally;
    int pend_ir;
    double pend_e;
    Part<R> out[MAXOUT];
    uint32_t out_pos[MAXOUT];     // parent's stream position at each push
    int nout;
    unsigned flags;
    int work;
    int tleft;                    // tstep-loop iterations left in this event
    int ncross, ndep, natom;
    __device__ R uni() { return rng.uni(); }
    // Consecutive deposits into one voxel are summed before the atomic.
    __device__ void deposit(int ir, R e) {
        ndep++;
        if (ir != pend_ir) {
            flush();
            pend_ir = ir;
        }
        pend_e += (double)e;
    }
    __device__ void flush() {
        if (pend_ir > 0 && pend_e != 0.0) {
            // the lanes of the warp that flush here together into the same
            // tally element (same voxel and tally slot) add once: the
            // group's sum, by its lowest lane (+4-5 % on the served beamlet
            // load and the slab beam over one atomic per lane)
            double *dst = &tally[pend_ir - 1];
            const unsigned act = __activemask();
            const unsigned grp = __match_any_sync(act, (unsigned long long)dst);
            const int lane = threadIdx.x & 31;
            double tot = pend_e;
            if (grp != (1u << lane)) {
                tot = 0.0;
                for (unsigned m = grp; m; m &= m - 1) tot += __shfl_sync(grp, pend_e, __ffs(m) - 1);
            }
            if (lane == __ffs(grp) - 1) {
                atomicAdd(dst, tot);
                natom++;
            }
        }
        pend_e = 0.0;
        pend_ir = -1;
    }
    __device__ void cross() { ncross++; }
    __device__ bool tstep_take() { return tleft-- > 0; }
    __device__ bool push(const Part<R> &q) { return push_at(q, rng.position()); }
    // A push made at stream position `pos` (an event run out of line).
    __device__ bool push_at(const Part<R> &q, uint32_t pos) {
        if (nout >= MAXOUT) {
            flags |= ERR_STACK;
            return false;
        }
        // static indices keep the outputs in registers
#pragma unroll
        for (int k = 0; k < MAXOUT; k++)
            if (k == nout) {
                out_pos[k] = pos;
                out[k] = q;
            }
        nout++;
        return true;
    }
    __device__ void err(unsigned f) { flags |= f; }
    __device__ bool tick() { return ++work < EV_BUDGET; }
};

// A photon event through the out-of-line photon_event_outline: its results
// folded back into the event environment in the order the photon step
// itself would have made them (stream, counters, deposit, pushed product).
template <int MAXOUT, typename R>
__device__ __forceinline__ bool photon_event(const DevData<R> &D, EvEnv<MAXOUT, R> &g, Part<R> &p) {
    const PhotonEventOut<R> o = photon_event_outline<R>(D, p, g.rng, g.work, EV_BUDGET);
    p = o.p;
    g.rng = o.e.rng;
    g.work = o.e.work;
    g.ncross += o.e.ncross;
    g.flags |= o.e.flags;
    if (o.e.dep_ir >= 0) g.deposit(o.e.dep_ir, o.e.dep_e);
    if (o.e.nq) g.push_at(o.e.q, o.e.qpos);
    return o.alive != 0;
}

template <typename R = float>
struct SrcEnv {
    Philox<R> rng;
    __device__ R uni() { return rng.uni(); }
};

// A queued particle is read once and written once per event, so its loads
// and stores bypass L1 and are marked streaming (evict first) in L2, which
// keeps the caches for the tables, the tallies and the kernels' local frames.
__device__ __forceinline__ void qload(const Queue &q, int i, Part<float> &p, int &tag, uint32_t &k0, uint32_t &k1,
                                      uint32_t &ctr) {
    const float4 a = __ldcs(&q.pos[i]);
    const float4 b = __ldcs(&q.dir[i]);
    const uint4 c = __ldcs(&q.id[i]);
    ctr = __ldcs(&q.ctr[i]);
    p.x = a.x; p.y = a.y; p.z = a.z; p.u = a.w;
    p.v = b.x; p.w = b.y; p.e = b.z; p.wt = b.w;
    p.ir = (int)c.x;
    tag = (int)c.y;
    p.iq = (tag & 3) - 1;
    k0 = c.z; k1 = c.w;
}

__device__ __forceinline__ void qload(const QueueT<double> &q, int i, Part<double> &p, int &tag, uint32_t &k0,
                                      uint32_t &k1, uint32_t &ctr) {
    const double2 *pa = (const double2 *)&q.pos[i], *pb = (const double2 *)&q.dir[i];
    const double2 a0 = __ldcs(pa), a1 = __ldcs(pa + 1), b0 = __ldcs(pb), b1 = __ldcs(pb + 1);
    const uint4 c = __ldcs(&q.id[i]);
    ctr = __ldcs(&q.ctr[i]);
    p.x = a0.x; p.y = a0.y; p.z = a1.x; p.u = a1.y;
    p.v = b0.x; p.w = b0.y; p.e = b1.x; p.wt = b1.y;
    p.ir = (int)c.x;
    tag = (int)c.y;
    p.iq = (tag & 3) - 1;
    k0 = c.z; k1 = c.w;
}

// sp/sr: splitting state, stored where the queue has it (photon queues of
// splitting engines); -1 = a photon not yet split.
__device__ __forceinline__ void qstore(const Queue &q, int i, const Part<float> &p, int slot, uint32_t k0, uint32_t k1,
                                       uint32_t ctr, int sp = -1, float sr = 0.f) {
    __stcs(&q.pos[i], make_float4(p.x, p.y, p.z, p.u));
    __stcs(&q.dir[i], make_float4(p.v, p.w, p.e, p.wt));
    __stcs(&q.id[i], make_uint4((uint32_t)p.ir, (uint32_t)((p.iq + 1) | (slot << 2)), k0, k1));
    __stcs(&q.ctr[i], ctr);
    if (q.sp) {
        q.sp[i] = sp;
        q.sr[i] = sr;
    }
}

__device__ __forceinline__ void qstore(const QueueT<double> &q, int i, const Part<double> &p, int slot, uint32_t k0,
                                       uint32_t k1, uint32_t ctr, int sp = -1, float sr = 0.f) {
    double2 *pa = (double2 *)&q.pos[i], *pb = (double2 *)&q.dir[i];
    __stcs(pa, make_double2(p.x, p.y));
    __stcs(pa + 1, make_double2(p.z, p.u));
    __stcs(pb, make_double2(p.v, p.w));
    __stcs(pb + 1, make_double2(p.e, p.wt));
    __stcs(&q.id[i], make_uint4((uint32_t)p.ir, (uint32_t)((p.iq + 1) | (slot << 2)), k0, k1));
    __stcs(&q.ctr[i], ctr);
    if (q.sp) {
        q.sp[i] = sp;
        q.sr[i] = sr;
    }
}

// Slot of a warp-aggregated append to `q` for the lanes with `want`: from
// the bottom, or from the top for lanes with `hi`; -1 for the other lanes
// (or on overflow, flagged).
template <typename Q>
__device__ __forceinline__ int warp_append(const Q &q, bool want, bool hi, unsigned active, unsigned &flags) {
    const int lane = threadIdx.x & 31;
    const unsigned mlo = __ballot_sync(active, want && !hi);
    const unsigned mhi = __ballot_sync(active, want && hi);
    int blo = 0, bhi = 0;
    if (mlo) {
        int leader = __ffs(mlo) - 1;
        if (lane == leader) blo = atomicAdd(q.count, __popc(mlo));
        blo = __shfl_sync(active, blo, leader);
    }
    if (mhi) {
        int leader = __ffs(mhi) - 1;
        if (lane == leader) bhi = atomicAdd(q.count_hi, __popc(mhi));
        bhi = __shfl_sync(active, bhi, leader);
    }
    if (!want) return -1;
    int k = hi ? bhi + __popc(mhi & lanemask_lt()) : blo + __popc(mlo & lanemask_lt());
    if (k >= q.cap) {
        flags |= ERR_QUEUE;
        return -1;
    }
    return hi ? q.cap - 1 - k : k;
}

// Entries of a queue (both ends) and the index of the f-th, top end first.
template <typename Q>
__device__ __forceinline__ int queue_size(const Q &q) {
    return min(min(*q.count, q.cap) + min(*q.count_hi, q.cap), q.cap);
}
template <typename Q>
__device__ __forceinline__ int queue_index(const Q &q, int f) {
    int nhi = min(*q.count_hi, q.cap);
    return f < nhi ? q.cap - 1 - f : f - nhi;
}

// Route the event's surviving particle and its secondaries to the output
// queues.  A secondary's stream key is derived from its parent's key, the
// parent's stream position when it was created and its index among the
// event's secondaries.  All 32 lanes of the warp take part (lanes without a
// particle pass alive = false, nout = 0).  The survivor keeps its splitting
// state (sp, sr); secondaries start unsplit.  Photons of zero weight (lost
// a Russian roulette) would deposit nothing and are not queued, and an
// electron at or below its region's cut-off is not queued either: its
// first event would only deposit its kinetic energy where it stands (the
// entry test of electron_step, which the drain applies to the same
// particle), so that deposit is made here.  It draws no random number, so
// trajectories do not change.  Returns the particles this lane queued.
template <int MAXOUT, bool DEFER = false, typename R = float>
__device__ __forceinline__ int emit(const DevData<R> &D, const QueueT<R> &outP, const QueueT<R> &outE, bool alive,
                                    const Part<R> &p, EvEnv<MAXOUT, R> &g, int slot, uint32_t k0, uint32_t k1,
                                    float esplit, int sp = -1, float sr = 0.f, const QueueT<R> *outI = nullptr,
                                    bool defer = false) {
    const unsigned full = 0xffffffffu;
    uint64_t pkey = ((uint64_t)k1 << 32) | k0;
    int queued = 0;
#pragma unroll
    for (int k = 0; k < 1 + MAXOUT; k++) {
        bool has;
        Part<R> q;
        uint32_t a0 = k0, a1 = k1, ac;
        if (k == 0) {
            has = alive;
            q = p;
            ac = g.rng.position();
        } else {
            has = k - 1 < g.nout;
            q = g.out[k - 1];
            uint64_t ck = mix64(pkey * 0x9E3779B97F4A7C15ull + ((uint64_t)g.out_pos[k - 1] << 1) + 1u +
                                ((uint64_t)(k - 1) << 40));
            a0 = (uint32_t)ck;
            a1 = (uint32_t)(ck >> 32);
            ac = 0;
        }
        if (__ballot_sync(full, has) == 0) continue;
        if (has && !(q.e == q.e && q.x == q.x && q.u == q.u)) {
            g.flags |= ERR_NAN;
            has = false;
        }
        if (has && q.iq == 0 && q.wt == R(0)) has = false;
        // an electron left at its discrete interaction goes to the
        // interaction queue
        const bool toi = DEFER && k == 0 && defer;
        bool isph = has && q.iq == 0 && !toi;
        bool isel = has && q.iq != 0 && !toi;
        if (isel && q.iq < 0 && q.e <= ecut_of(D, q.ir)) {
            g.deposit(q.ir, q.wt * (q.e - R(D_RM)));
            isel = false;
        }
        int ip = warp_append(outP, isph, false, full, g.flags);
        int ie = warp_append(outE, isel, esplit > 0.f && q.e > (R)esplit, full, g.flags);
        if (ip >= 0) qstore(outP, ip, q, slot, a0, a1, ac, k == 0 ? sp : -1, k == 0 ? sr : 0.f);
        if (ie >= 0) qstore(outE, ie, q, slot, a0, a1, ac);
        queued += (ip >= 0) + (ie >= 0);
        if (DEFER && k == 0) {
            int ii = warp_append(*outI, has && toi, false, full, g.flags);
            if (ii >= 0) qstore(*outI, ii, q, slot, a0, a1, ac);
            queued += ii >= 0;
        }
    }
    g.flush();
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

// One event of a split photon (photon splitting, ompmc.c:1867-2139 with
// nsplit > 1).  A queued photon is a ray of nsplit sub-photons of weight
// wt/nsplit whose interaction sites are stratified along it.  Its first
// event checks the cut-off, draws the stratification offset r and the
// surviving sub-photon, and sets the ray's weight; every event then moves
// one sub-photon, k, from the previous site by its share of mean free
// paths, ln(eta_{k-1} / eta_k) with eta_k = (nsplit - k - r) / nsplit
// (eta_{-1} = 1), and samples its interaction.  The charged products are
// pushed with the sub-photon's weight; the scattered photon of the
// surviving sub-photon is pushed with the full weight (as a new, unsplit
// photon) and the others' are dropped.  p becomes the ray at the site;
// returns true while it has sub-photons left.  The draws differ from the
// plain form's order (one stream per ray), the sampled distribution is the
// same.
template <typename R, typename Env>
__device__ __forceinline__ bool split_event(const DevData<R> &D, Env &g, Part<R> &p, int &sp, float &sr) {
    const int ns = D.nsplit;
    if (sp < 0) {
        if (p.e <= pcut_of(D, p.ir) || p.wt == 0.f) {
            g.deposit(p.ir, p.wt * p.e);
            return false;
        }
        sr = g.uni();
        int isurv = (int)(g.uni() * (float)ns);
        sp = min(isurv, ns - 1);
        p.wt = p.wt / (float)ns;
    }
    const int isplit = sp >> 16, isurv = sp & 0xffff;
    const float den = (float)(ns - isplit) - sr;
    if (den <= 0.f) return false;
    const float num = isplit == 0 ? (float)ns : den + 1.f;
    const float dpmfp = m_log(num / den);
    const float gle = m_log(p.e);
    Part<float> q = p;
    q.iq = 0;
    int imed, lgle;
    float cohfac;
    if (!photon_walk(D, g, q, gle, dpmfp, imed, lgle, cohfac)) return false;
    p.x = q.x; p.y = q.y; p.z = q.z;
    p.ir = q.ir;
    const bool surv = isplit == isurv;
    if (g.uni() <= 1.f - cohfac) {
        if (surv) {
            q.wt *= (float)ns;
            rayleigh(D, g, q, imed, gle, lgle);
            g.push(q);
        }
    } else {
        photon_interact(D, g, q, p.e, gle, imed, lgle);
        // the interaction pushed at most one product; keep it and q as the
        // splitting rules say
        if (g.nout == 1 && g.out[0].iq == 0) {
            if (surv) g.out[0].wt *= (float)ns;
            else g.nout = 0;
        }
        if (q.iq != 0 || surv) {
            if (q.iq == 0) q.wt *= (float)ns;
            g.push(q);
        }
    }
    sp = ((isplit + 1) << 16) | isurv;
    return isplit + 1 < ns;
}

// Events of one queue.  Warps take 32 particles at a time from a counter,
// so work is balanced between warps however long their events run.
// KIND: EV_PHOTON, EV_ELECTRON, EV_SPLIT (photons of a splitting engine)
// or EV_INTERACT (electrons at their discrete interaction, with
// D.defer_interact).  `qi`: the interaction queue (EV_ELECTRON with
// D.defer_interact appends there).
enum { EV_PHOTON = 0, EV_ELECTRON = 1, EV_SPLIT = 2, EV_INTERACT = 3, EV_ELECTRON_DEFER = 4 };
template <int KIND, typename R = float>
__device__ __forceinline__ void transport_events(const DevData<R> &D, const QueueT<R> &in, const QueueT<R> &outP,
                                                 const QueueT<R> &outE, double *tallies, long nvox, Ctl *ctl,
                                                 uint32_t seedw, ServeDev *sd, int nbmax, const QueueT<R> &qi) {
    constexpr int MAXOUT = KIND == EV_SPLIT ? EV_MAXOUT_SPLIT : EV_MAXOUT;
    const unsigned full = 0xffffffffu;
    constexpr bool ELECTRON = KIND == EV_ELECTRON || KIND == EV_ELECTRON_DEFER;
    const int kq = ELECTRON ? 1 : (KIND == EV_INTERACT ? 2 : 0);
    const int ks = KIND == EV_PHOTON || KIND == EV_SPLIT ? 0 : 1;   // counters: photon or electron
    const int n = queue_size(in);
    const int tsteps = ctl->tsteps;
    const float esplit = ctl->esplit;
    const int lane = threadIdx.x & 31;
    unsigned flags = 0;
    unsigned c_ev = 0, c_steps = 0, c_cross = 0, c_dep = 0, c_atom = 0;
    for (int guard = 0; guard < (1 << 26); guard++) {
        int base = 0;
        if (lane == 0) base = atomicAdd(&ctl->fetch[kq], 32);
        base = __shfl_sync(full, base, 0);
        if (base >= n) break;
        const bool valid = base + lane < n;
        const int i = valid ? queue_index(in, base + lane) : 0;
        Part<R> p;
        int tag = 0;
        uint32_t k0 = 0, k1 = 0, pos = 0;
        if (valid) qload(in, i, p, tag, k0, k1, pos);
        int sp = -1;
        float sr = 0.f;
        if (KIND == EV_SPLIT && valid) {
            sp = in.sp[i];
            sr = in.sr[i];
        }
        const int slot = tag >> 2;
        EvEnv<MAXOUT, R> g;
        g.rng.init(((uint64_t)k1 << 32) | k0, seedw, pos);
        g.tally = tallies + (long)slot * nvox;
        g.pend_ir = -1;
        g.pend_e = 0.0;
        g.nout = 0;
        g.flags = 0;
        g.work = 0;
        g.tleft = tsteps;
        g.ncross = g.ndep = g.natom = 0;
        bool alive = false, defer = false;
        if (valid) {
            if (KIND == EV_PHOTON) {
                alive = photon_event(D, g, p);
            } else if (ELECTRON) {
                int r = electron_step<R, EvEnv<MAXOUT, R>, KIND == EV_ELECTRON_DEFER>(D, g, p);
                alive = r != E_DEAD;
                defer = r == E_INTERACT;
            } else if constexpr (KIND == EV_SPLIT) {
                alive = split_event(D, g, p, sp, sr);
            } else {
                electron_interact(D, g, p);
                alive = true;
            }
            g.flush();
        }
        int emitted = KIND == EV_ELECTRON_DEFER
                          ? emit<MAXOUT, true, R>(D, outP, outE, alive, p, g, slot, k0, k1, esplit, sp, sr, &qi, defer)
                          : emit<MAXOUT, false, R>(D, outP, outE, alive, p, g, slot, k0, k1, esplit, sp, sr);
        if (sd) add_live(sd->live, nbmax, valid ? slot : 0, valid ? emitted - 1 : 0, full);
        flags |= g.flags;
        c_ev += valid;
        c_steps += g.work;
        c_cross += g.ncross;
        c_dep += g.ndep;
        c_atom += g.natom;
    }
    report_flags(ctl, flags, full);
    if (KIND != EV_INTERACT) report_count(&ctl->st_events[ks], c_ev, full);
    report_count(&ctl->st_steps[ks], c_steps, full);
    report_count(&ctl->st_cross[ks], c_cross, full);
    report_count(&ctl->st_dep[ks], c_dep, full);
    report_count(&ctl->st_atom[ks], c_atom, full);
}

// Photon events of the queued photons.  `live` (may be null) receives the
// change of each serving request's live-particle count.
template <typename R>
__global__ void __launch_bounds__(EV_MAX_BLOCK) k_photon_step(DevData<R> D, QueueT<R> in, QueueT<R> outP,
                                                     QueueT<R> outE, double *tallies, long nvox, Ctl *ctl,
                                                     uint32_t seedw, ServeDev *sd, int nbmax, QueueT<R> qi) {
    transport_events<EV_PHOTON, R>(D, in, outP, outE, tallies, nvox, ctl, seedw, sd, nbmax, qi);
}

// Photon events of a splitting engine (nsplit > 1): one sub-photon each.
__global__ void __launch_bounds__(EV_MAX_BLOCK) k_photon_split_step(DevData<float> D, Queue in, Queue outP,
                                                           Queue outE, double *tallies, long nvox, Ctl *ctl,
                                                           uint32_t seedw, ServeDev *sd, int nbmax, Queue qi) {
    transport_events<EV_SPLIT>(D, in, outP, outE, tallies, nvox, ctl, seedw, sd, nbmax, qi);
}

// Electron/positron events of the queued charged particles: at most the
// cycle's budget of tstep-loop iterations each, then the particle is
// re-queued.  The step is latency bound; the occupancy it is compiled for
// (electron_minb) trades resident warps against spilled local frames.
template <bool DEFER, typename R = float>
__global__ void __launch_bounds__(EV_MAX_BLOCK, electron_minb<R>())
    k_electron_step(DevData<R> D, QueueT<R> in, QueueT<R> outP, QueueT<R> outE, double *tallies, long nvox, Ctl *ctl,
                    uint32_t seedw, ServeDev *sd, int nbmax, QueueT<R> qi) {
    transport_events<DEFER ? EV_ELECTRON_DEFER : EV_ELECTRON, R>(D, in, outP, outE, tallies, nvox, ctl, seedw, sd,
                                                                  nbmax, qi);
}

// The electron kernel of the engine: interactions in a kernel of their own
// (D.defer_interact) or in place.
template <typename R = float>
static TransportKernelT<R> electron_kernel(const omc_engine *e) {
    return e->d32.d.defer_interact ? k_electron_step<true, R> : k_electron_step<false, R>;
}

// Discrete interactions of the electrons the electron kernel left at their
// interaction sites (D.defer_interact): the samplers run in a kernel of
// their own, so the transport kernel's code stays small.
template <typename R = float>
__global__ void __launch_bounds__(EV_MAX_BLOCK) k_electron_interact(DevData<R> D, QueueT<R> in, QueueT<R> outP,
                                                           QueueT<R> outE, double *tallies, long nvox, Ctl *ctl,
                                                           uint32_t seedw, ServeDev *sd, int nbmax, QueueT<R> qi) {
    transport_events<EV_INTERACT, R>(D, in, outP, outE, tallies, nvox, ctl, seedw, sd, nbmax, qi);
}

// ------------------------------------------------------------ drain
// Once every history is injected and few particles remain, transport
// cycles launch mostly idle kernels whose duration is the latency of their
// longest events, and each particle waits a whole cycle between events.
// The drain runs each remaining particle to the end of its sub-history in
// one launch instead: one thread per queued particle, its secondaries on a
// local stack.  Every particle keeps its own random stream and its
// secondaries get the keys emit() gives them, electrons run to their
// interaction without a budget (budgets do not change trajectories) and
// interactions are sampled in place (the same draws as the interaction
// kernel), so the dose is the one the cycles would have produced, up to
// the summation order of the FP64 tallies.  SPLIT: photons are split rays
// (nsplit > 1) whose state (next sub-photon, survivor, offset) rides on the
// stack with them, as in the photon queues.
constexpr int DRAIN_STACK = 48;
// 4 resident blocks of 128 per SM: up to 128 registers and no spills.  The
// drain's length is the latency of its longest sub-history in one thread,
// which spilled registers lengthen; it never needs more lanes than
// particles (1.2 % faster on slab64 than 8 blocks at 64 registers).
constexpr int DRAIN_BLOCK = 128;

template <typename R>
struct DrainPart {
    Part<R> p;
    uint32_t k0, k1, pos;
    int sp;       // splitting state (-1: not yet split)
    float sr;
};

// STATS (profiled runs): record the largest sub-history a thread ran.
template <bool SPLIT, bool STATS = false, typename R = float>
__global__ void __launch_bounds__(DRAIN_BLOCK, 4) k_drain(DevData<R> D, QueueT<R> qP, QueueT<R> qE, double *tallies,
                                                        long nvox, Ctl *ctl, uint32_t seedw) {
    constexpr int MAXOUT = SPLIT ? EV_MAXOUT_SPLIT : EV_MAXOUT;
    const int np = queue_size(qP), ne = queue_size(qE);
    const int n = np + ne;
    DrainPart<R> st[DRAIN_STACK];
    unsigned flags = 0;
    unsigned long long c_ev[2] = {0, 0}, c_steps[2] = {0, 0}, c_cross[2] = {0, 0}, c_dep[2] = {0, 0},
                       c_atom[2] = {0, 0};
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const QueueT<R> &q = t < np ? qP : qE;
        int tag = 0;
        const int qi = queue_index(q, t < np ? t : t - np);
        qload(q, qi, st[0].p, tag, st[0].k0, st[0].k1, st[0].pos);
        st[0].sp = (SPLIT && q.sp) ? q.sp[qi] : -1;
        st[0].sr = (SPLIT && q.sr) ? q.sr[qi] : 0.f;
        EvEnv<MAXOUT, R> g;
        g.tally = tallies + (long)(tag >> 2) * nvox;
        g.pend_ir = -1;
        g.pend_e = 0.0;
        g.flags = 0;
        g.natom = 0;
        int top = 0;
        // this sub-history: events, events of its first particle, steps
        int x_ev = 0, x_chain = 0, x_steps = 0;
        bool first_alive = true;
        for (int guard = 0; top >= 0; guard++) {
            const bool first = first_alive && top == 0;
            x_ev++;
            x_chain += first;
            if (guard > (1 << 22)) {
                g.flags |= ERR_LOOP;
                break;
            }
            DrainPart<R> &e = st[top];
            Part<R> p = e.p;
            const uint64_t pkey = ((uint64_t)e.k1 << 32) | e.k0;
            g.rng.init(pkey, seedw, e.pos);
            g.nout = 0;
            g.work = 0;
            g.tleft = 1 << 30;
            g.ncross = g.ndep = 0;
            const int kind = p.iq == 0 ? 0 : 1;
            int sp = e.sp;
            float sr = e.sr;
            bool alive;
            if (kind == 1) alive = electron_step<R, EvEnv<MAXOUT, R>, false>(D, g, p) == E_ALIVE;
            else if constexpr (SPLIT) alive = split_event(D, g, p, sp, sr);
            else alive = photon_event(D, g, p);
            c_ev[kind]++;
            x_steps += g.work;
            c_steps[kind] += g.work;
            c_cross[kind] += g.ncross;
            c_dep[kind] += g.ndep;
            if (alive && !(p.e == p.e && p.x == p.x && p.u == p.u)) {
                g.flags |= ERR_NAN;
                alive = false;
            }
            if (alive && p.iq == 0 && p.wt == R(0)) alive = false;
            if (alive) {
                e.p = p;
                e.pos = g.rng.position();
                e.sp = sp;
                e.sr = sr;
            } else {
                top--;
                first_alive = first_alive && !first;
            }
            for (int k = 0; k < g.nout; k++) {
                const Part<R> &s2 = g.out[k];
                if (!(s2.e == s2.e && s2.x == s2.x && s2.u == s2.u)) {
                    g.flags |= ERR_NAN;
                    continue;
                }
                if (s2.iq == 0 && s2.wt == R(0)) continue;
                if (top + 1 >= DRAIN_STACK) {
                    g.flags |= ERR_STACK;
                    continue;
                }
                uint64_t ck = mix64(pkey * 0x9E3779B97F4A7C15ull + ((uint64_t)g.out_pos[k] << 1) + 1u +
                                    ((uint64_t)k << 40));
                top++;
                st[top].p = s2;
                st[top].k0 = (uint32_t)ck;
                st[top].k1 = (uint32_t)(ck >> 32);
                st[top].pos = 0;
                st[top].sp = -1;
                st[top].sr = 0.f;
            }
        }
        g.flush();
        if (STATS) {
            atomicMax(&ctl->drain_max_events, x_ev);
            atomicMax(&ctl->drain_max_chain, x_chain);
            atomicMax(&ctl->drain_max_steps, x_steps);
        }
        c_atom[1] += g.natom;     // tally atomics of the whole sub-history
        flags |= g.flags;
    }
    if (flags) atomicOr(&ctl->flags, flags);
    for (int k = 0; k < 2; k++) {
        if (c_ev[k]) atomicAdd(&ctl->st_events[k], c_ev[k]);
        if (c_steps[k]) atomicAdd(&ctl->st_steps[k], c_steps[k]);
        if (c_cross[k]) atomicAdd(&ctl->st_cross[k], c_cross[k]);
        if (c_dep[k]) atomicAdd(&ctl->st_dep[k], c_dep[k]);
        if (c_atom[k]) atomicAdd(&ctl->st_atom[k], c_atom[k]);
    }
}

template <typename R = float>
__global__ void k_source(DevData<R> D, BeamSrc<R> S, QueueT<R> qP, QueueT<R> qE, Ctl *ctl, long long nper,
                         uint64_t seed, uint32_t seedw) {
    int n = ctl->inject;
    long long base = ctl->hist_base;
    double es = 0;
    unsigned flags = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        unsigned active = __activemask();
        long long h = base + i;
        SrcEnv<R> g;
        uint64_t key = mix64(seed ^ (uint64_t)h * 0x9E3779B97F4A7C15ull);
        g.rng.init(key, seedw);
        R ein;
        Part<R> p = beam_primary(D, S, g, ein);
        es += ein;
        int slot = (int)(h / nper);
        int ip = warp_append(qP, p.iq == 0, false, active, flags);
        int ie = warp_append(qE, p.iq != 0, ctl->esplit > 0.f && p.e > (R)ctl->esplit, active, flags);
        if (ip >= 0) qstore(qP, ip, p, slot, (uint32_t)key, (uint32_t)(key >> 32), g.rng.position());
        if (ie >= 0) qstore(qE, ie, p, slot, (uint32_t)key, (uint32_t)(key >> 32), g.rng.position());
    }
    for (int o = 16; o > 0; o >>= 1) es += __shfl_down_sync(0xffffffffu, es, o);
    if ((threadIdx.x & 31) == 0 && es != 0.0) atomicAdd(&ctl->src_energy, es);
    unsigned active = __activemask();
    report_flags(ctl, flags, active);
}

// Electron budget of a cycle whose electron queue holds nE particles on a
// GPU with `lanes` resident threads: the base budget while the queue fills
// the GPU, multiplied by up to `boost` as it drains (the drain tail then
// takes few cycles; a lane's events of any length give the same result).
__device__ __forceinline__ void plan_budget(Ctl *ctl, long long nE, const PlanCfg &c) {
    long long me = 1;
    if (c.boost > 1 && nE < c.lanes) {
        me = c.lanes / (nE > 0 ? nE : 1);
        me = me > c.boost ? c.boost : me;
    }
    ctl->tsteps = (int)(c.tsteps * me);
    ctl->esplit = c.esplit;
    ctl->fetch[0] = 0;
    ctl->fetch[1] = 0;
    ctl->fetch[2] = 0;
    ctl->cnt_int = 0;
    ctl->cnt_int_hi = 0;
}

// Particles in the cycle's input queues; an overflow of either (the two
// ends met) is flagged.  The output queues (the previous cycle's inputs,
// all consumed) are emptied.
__device__ __forceinline__ void plan_queues(Ctl *ctl, int iph, int iel, int cap, long long &np, long long &ne) {
    np = (long long)ctl->cnt[iph] + ctl->cnt_hi[iph];
    ne = (long long)ctl->cnt[iel] + ctl->cnt_hi[iel];
    if (np > cap || ne > cap) ctl->flags |= ERR_QUEUE;
    np = np > cap ? cap : np;
    ne = ne > cap ? cap : ne;
    ctl->cnt[iph ^ 2] = 0;
    ctl->cnt[iel ^ 2] = 0;
    ctl->cnt_hi[iph ^ 2] = 0;
    ctl->cnt_hi[iel ^ 2] = 0;
}

// Histories to inject this cycle: keep `target` particles in flight (a
// photon of a splitting engine counts nsplit times).  Also
// sets the cycle's electron budget and empties the output queues (the
// previous cycle's inputs, all consumed).
__global__ void k_plan(Ctl *ctl, int iph, int iel, PlanCfg c) {
    long long np, ne;
    plan_queues(ctl, iph, iel, c.cap, np, ne);
    long long rem = ctl->hist_total - ctl->hist_next;
    long long inj = (c.target - (np * c.pweight + ne)) / c.pweight;
    if (inj < 0) inj = 0;
    if (inj > rem) inj = rem;
    long long room = (long long)c.cap - (np > ne ? np : ne);
    if (inj > room) inj = room > 0 ? room : 0;
    ctl->inject = (int)inj;
    ctl->hist_base = ctl->hist_next;
    ctl->hist_next += inj;
    plan_budget(ctl, ne, c);
}

// ------------------------------------------------------------------ host
// The event state of precision R: the FP32 form's or the FP64 form's.
template <typename R>
EventStateT<R> *&state_of(omc_engine *e);
template <>
EventStateT<float> *&state_of<float>(omc_engine *e) {
    return e->ev;
}
template <>
EventStateT<double> *&state_of<double>(omc_engine *e) {
    return e->ev64;
}
template <typename R>
const EventStateT<R> &state(const omc_engine *e) {
    return *state_of<R>(const_cast<omc_engine *>(e));
}

// Tables and flags the event kernels of precision R run with.  The FP64
// event form uses the FP64 tables with the event form's options (re-drawn
// interaction distance, deferred interactions, delta tracking) instead of
// the plain form's.
template <typename R>
DevData<R> event_data(const omc_engine *e);
template <>
DevData<float> event_data<float>(const omc_engine *e) {
    return e->d32.d;
}
template <>
DevData<double> event_data<double>(const omc_engine *e) {
    DevData<double> d = e->d64.d;
    d.chsteps = e->d32.d.chsteps;
    d.defer_interact = e->d32.d.defer_interact;
    d.woodcock = d.uniform && e->d32.d.woodcock ? 1 : 0;
    d.nsplit = 1;
    return d;
}

template <typename R>
static int alloc_queue(omc_engine *e, DBuf &b, QueueT<R> &q, int cap, int *count, int *count_hi) {
    // pos and dir: 4 values of R each; id: 16 bytes; ctr: 4 bytes (every
    // array starts on a 16-byte boundary for any cap)
    const size_t v4 = (size_t)cap * 4 * sizeof(R), per = (size_t)cap * 4;
    int rc = b.alloc(2 * v4 + 5 * per);
    if (rc) return set_err(e, rc, "event queue allocation failed");
    char *p = (char *)b.p;
    q.pos = (typename QVec<R>::T *)p;
    q.dir = (typename QVec<R>::T *)(p + v4);
    q.id = (uint4 *)(p + 2 * v4);
    q.ctr = (uint32_t *)(p + 2 * v4 + 4 * per);
    q.count = count;
    q.count_hi = count_hi;
    q.cap = cap;
    q.sp = nullptr;
    q.sr = nullptr;
    return OMC_OK;
}

// The photon kernel of the engine: split photons when nsplit > 1 (FP32
// form only).
template <typename R = float>
static TransportKernelT<R> photon_kernel(const omc_engine *e);
template <>
TransportKernelT<float> photon_kernel<float>(const omc_engine *e) {
    return e->d32.d.nsplit > 1 ? k_photon_split_step : k_photon_step<float>;
}
template <>
TransportKernelT<double> photon_kernel<double>(const omc_engine *) {
    return k_photon_step<double>;
}

// Resident blocks per SM of the transport kernels -> one-wave grids.
template <typename R>
static void size_grids(omc_engine *e, EventStateT<R> &S) {
    int bp = 0, be = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bp, photon_kernel<R>(e), S.block, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&be, electron_kernel<R>(e), S.block, 0);
    S.grid_p = e->sm_count * std::max(1, bp);
    S.grid_e = e->sm_count * std::max(1, be);
    int bi = 0, bd = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bi, k_electron_interact<R>, S.block, 0);
    S.grid_i = e->sm_count * std::max(1, bi);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bd, k_drain<false, false, R>, DRAIN_BLOCK, 0);
    S.drain_lanes = e->sm_count * std::max(1, bd) * DRAIN_BLOCK;
    S.lanes = S.grid_e * S.block;
}

// The interaction queue, allocated when the engine first needs it.
template <typename R>
static int event_interact_queue_t(omc_engine *e) {
    EventStateT<R> &S = *state_of<R>(e);
    if (!e->d32.d.defer_interact || S.int_buf.p) return OMC_OK;
    return alloc_queue(e, S.int_buf, S.qi, S.cap, &S.ctl_d->cnt_int, &S.ctl_d->cnt_int_hi);
}
int event_interact_queue(omc_engine *e) { return event_interact_queue_t<float>(e); }

template <typename R>
static int event_prepare_t(omc_engine *e) {
    EventStateT<R> *&sp = state_of<R>(e);
    if (sp && sp->ready) return OMC_OK;
    if (!sp) sp = new EventStateT<R>();
    EventStateT<R> &S = *sp;
    long cap = e->opt.queue_capacity > 0 ? e->opt.queue_capacity : (1L << 22);
    S.cap = (int)std::min(cap, (long)(1L << 30));
    // warps fetch work 32 particles at a time: whole warps per block, at
    // most the transport kernels' launch bound
    S.block = e->opt.block > 0 ? std::min(EV_MAX_BLOCK, (e->opt.block + 31) / 32 * 32) : 256;
    S.grid = e->sm_count * std::max(1, 2048 / S.block);
    size_grids(e, S);
    // 1 measured best on the slab workload while the queues are full (with
    // the default electron_chsteps = 3: at most three CH steps per event)
    S.tsteps = e->opt.electron_tsteps > 0 ? e->opt.electron_tsteps : 1;
    S.boost = e->opt.tail_boost > 0 ? e->opt.tail_boost : 32;
    S.inflight = e->opt.inflight > 0 ? e->opt.inflight : (1LL << 20);
    S.esplit = e->opt.electron_split > 0 ? e->opt.electron_split + D_RM : 0.0;
    int rc = S.ctl.alloc(sizeof(Ctl));
    if (rc) return set_err(e, rc, "control block allocation failed");
    S.ctl_d = S.ctl.template as<Ctl>();
    for (int i = 0; i < 4; i++)
        if ((rc = alloc_queue(e, S.buf[i], S.q[i], S.cap, &S.ctl_d->cnt[i], &S.ctl_d->cnt_hi[i]))) return rc;
    if (e->d32.d.nsplit > 1 && sizeof(R) == 4) {
        // splitting state of the two photon queues (A and B)
        for (int k = 0; k < 2; k++) {
            size_t per = (size_t)S.cap * 4;
            if ((rc = S.split_buf[k].alloc(per * 2))) return set_err(e, rc, "splitting state allocation failed");
            QueueT<R> &q = S.q[2 * k];
            q.sp = S.split_buf[k].template as<int>();
            q.sr = (float *)((char *)S.split_buf[k].p + per);
        }
    }
    if (cudaStreamCreateWithFlags(&S.side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&S.fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&S.join, cudaEventDisableTiming) != cudaSuccess)
        return set_err(e, OMC_E_DEVICE, "side stream creation failed");
    S.ready = true;
    return OMC_OK;
}
int event_prepare(omc_engine *e) { return event_prepare_t<float>(e); }

// The transport kernels of one cycle after its source kernel.  Profiled
// (`ev`): one after the other on the engine's stream, an event after each.
// Otherwise (captured into the cycle graphs) the photon kernel runs on the
// side stream beside the electron kernels: they read different input
// queues and append to the output queues, the tallies and the counters
// with atomics only.  Launched after the electron kernel, its blocks take
// the SMs that the electron kernel's last blocks leave (4-5 % faster on
// slab64; same dose).  The side stream joins the engine's stream before the
// next cycle.
template <typename R = float>
static void launch_transport(omc_engine *e, int iph, int iel, int oph, int oel, double *tallies, uint32_t seedw,
                             ServeDev *sd, int nbmax, cudaEvent_t *ev) {
    EventStateT<R> &S = *state_of<R>(e);
    const long nvox = e->ph.nvox();
    const DevData<R> D = event_data<R>(e);
    auto photons = [&](cudaStream_t st) {
        photon_kernel<R>(e)<<<S.grid_p, S.block, 0, st>>>(D, S.q[iph], S.q[oph], S.q[oel], tallies, nvox, S.ctl_d,
                                                          seedw, sd, nbmax, S.qi);
    };
    auto electrons = [&]() {
        electron_kernel<R>(e)<<<S.grid_e, S.block, 0, e->stream>>>(D, S.q[iel], S.q[oph], S.q[oel], tallies, nvox,
                                                                    S.ctl_d, seedw, sd, nbmax, S.qi);
        if (D.defer_interact)
            k_electron_interact<R><<<S.grid_i, S.block, 0, e->stream>>>(D, S.qi, S.q[oph], S.q[oel], tallies, nvox,
                                                                        S.ctl_d, seedw, sd, nbmax, S.qi);
    };
    if (ev || !S.side) {
        photons(e->stream);
        if (ev) cudaEventRecord(ev[3], e->stream);
        electrons();
        return;
    }
    cudaEventRecord(S.fork, e->stream);
    cudaStreamWaitEvent(S.side, S.fork, 0);
    electrons();
    photons(S.side);
    cudaEventRecord(S.join, S.side);
    cudaStreamWaitEvent(e->stream, S.join, 0);
}

// Event-form tuning parameters of an engine (values <= 0 keep the current
// one); the queues are not reallocated.
int event_set_params(omc_engine *e, int tsteps, int boost, long long inflight, int block, double split_kinetic) {
    if (tsteps > 0) e->opt.electron_tsteps = tsteps;
    if (boost > 0) e->opt.tail_boost = boost;
    if (inflight > 0) e->opt.inflight = inflight;
    if (split_kinetic >= 0) e->opt.electron_split = split_kinetic;
    if (block > 0) {
        if (block % 32 || block > EV_MAX_BLOCK)
            return set_err(e, OMC_E_ARG, "block must be a multiple of 32, at most 256");
        e->opt.block = block;
    }
    auto apply = [&](auto &S) {
        S.tsteps = e->opt.electron_tsteps > 0 ? e->opt.electron_tsteps : 1;
        S.boost = e->opt.tail_boost > 0 ? e->opt.tail_boost : 32;
        S.inflight = e->opt.inflight > 0 ? e->opt.inflight : (1LL << 20);
        S.esplit = e->opt.electron_split > 0 ? e->opt.electron_split + D_RM : 0.0;
        S.block = e->opt.block > 0 ? std::min(EV_MAX_BLOCK, e->opt.block) : 256;
        S.grid = e->sm_count * std::max(1, 2048 / S.block);
        size_grids(e, S);
    };
    if (e->ev && e->ev->ready) apply(*e->ev);
    if (e->ev64 && e->ev64->ready) apply(*e->ev64);
    return OMC_OK;
}

template <typename R>
static PlanCfg plan_cfg_t(const omc_engine *e, long long target) {
    const EventStateT<R> &S = state<R>(e);
    PlanCfg c;
    c.target = target;
    c.cap = S.cap;
    c.lanes = S.lanes;
    c.boost = S.boost;
    c.tsteps = S.tsteps;
    c.esplit = (float)S.esplit;
    c.pweight = sizeof(R) == 4 ? std::max(1, e->d32.d.nsplit) : 1;
    return c;
}
PlanCfg plan_cfg(const omc_engine *e, long long target) { return plan_cfg_t<float>(e, target); }

void event_release(omc_engine *e) {
    delete e->ev;
    e->ev = nullptr;
    delete e->ev64;
    e->ev64 = nullptr;
}

// One transport cycle with input buffers `in` (0 = A, 1 = B).  With `ev`
// (profiling) the launches are sequential and an event is recorded before
// each and after the last.
template <typename R = float>
static void launch_cycle(omc_engine *e, int in, const BeamSrc<R> &src, double *tallies, long nper, uint64_t seed,
                         long long target, cudaEvent_t *ev = nullptr) {
    EventStateT<R> &S = *state_of<R>(e);
    int iph = in == 0 ? 0 : 2, iel = iph + 1;
    int oph = in == 0 ? 2 : 0, oel = oph + 1;
    uint32_t seedw = (uint32_t)(seed >> 32);
    if (ev) cudaEventRecord(ev[0], e->stream);
    k_plan<<<1, 1, 0, e->stream>>>(S.ctl_d, iph, iel, plan_cfg_t<R>(e, target));
    if (ev) cudaEventRecord(ev[1], e->stream);
    k_source<R><<<S.grid, S.block, 0, e->stream>>>(event_data<R>(e), src, S.q[iph], S.q[iel], S.ctl_d, nper, seed,
                                                   seedw);
    if (ev) cudaEventRecord(ev[2], e->stream);
    launch_transport<R>(e, iph, iel, oph, oel, tallies, seedw, nullptr, 1, ev);
    if (ev) cudaEventRecord(ev[4], e->stream);
}

// Particles left in the queues at or below which the transport switches
// from cycles to the drain (0: never).  By default half of the drain
// kernel's resident threads (≈38 k): the drain serialises each particle's
// whole remaining cascade in one thread, so it pays only once the cycles
// are mostly idle (measured on slab64: ≈40 k best of 5 k - 1 M particles,
// for 10^6- and 10^7-history runs alike).
template <typename R>
static long long drain_threshold_t(const omc_engine *e) {
    const EventStateT<R> &S = state<R>(e);
    if (e->opt.drain_particles < 0) return 0;
    return e->opt.drain_particles > 0 ? e->opt.drain_particles : S.drain_lanes / 2;
}
long long drain_threshold(const omc_engine *e) { return drain_threshold_t<float>(e); }

// The drain over the queues `iph`/`iph + 1` holding `left` particles, on
// the streams of the cycles that filled them (seed word `seedw`); `stats`
// records its largest sub-history.
template <typename R = float>
static void launch_drain(omc_engine *e, int iph, long long left, double *tallies, uint32_t seedw,
                         bool stats = false) {
    EventStateT<R> &S = *state_of<R>(e);
    long long g = (left + DRAIN_BLOCK - 1) / DRAIN_BLOCK;
    g = std::max(1LL, std::min(g, (long long)S.drain_lanes / DRAIN_BLOCK * 4));
    const DevData<R> D = event_data<R>(e);
    void (*kd)(DevData<R>, QueueT<R>, QueueT<R>, double *, long, Ctl *, uint32_t);
    if constexpr (sizeof(R) == 4)
        kd = D.nsplit > 1 ? (stats ? k_drain<true, true, R> : k_drain<true, false, R>)
                          : (stats ? k_drain<false, true, R> : k_drain<false, false, R>);
    else
        kd = stats ? k_drain<false, true, R> : k_drain<false, false, R>;
    kd<<<(int)g, DRAIN_BLOCK, 0, e->stream>>>(D, S.q[iph], S.q[iph + 1], tallies, e->ph.nvox(), S.ctl_d, seedw);
}

// Profiled transport: cycles launched one by one with events around each
// kernel; per-kernel device time accumulated into S.prof, one trace row per
// cycle.
static int run_profiled(omc_engine *e, const BeamSrc<float> &src, double *tallies, long nper, uint64_t seed,
                        long long target, Ctl &h, long &cycles) {
    EventState &S = *e->ev;
    for (auto &p : S.prof) p = KernelProfile();
    S.trace.clear();
    for (double &v : S.drain_stats) v = 0;
    cudaEvent_t ev[5];
    for (auto &x : ev) cudaEventCreate(&x);
    int rc = OMC_OK;
    cycles = 0;
    int cnt_in[2] = {0, 0};   // queue sizes the cycle starts with (before injection)
    for (;;) {
        int in = (int)(cycles & 1);
        launch_cycle(e, in, src, tallies, nper, seed, target, ev);
        cycles++;
        if ((rc = cuda_check(e, cudaEventSynchronize(ev[4]), "profiled cycle"))) break;
        float t[4];
        for (int k = 0; k < 4; k++) cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]);
        cudaMemcpy(&h, S.ctl_d, sizeof(Ctl), cudaMemcpyDeviceToHost);
        int oph = in == 0 ? 2 : 0;
        double row[6] = {(double)h.inject, (double)cnt_in[0] + h.inject, (double)cnt_in[1], t[1], t[2], t[3]};
        S.trace.insert(S.trace.end(), row, row + 6);
        cnt_in[0] = std::min(h.cnt[oph] + h.cnt_hi[oph], S.cap);
        cnt_in[1] = std::min(h.cnt[oph + 1] + h.cnt_hi[oph + 1], S.cap);
        S.prof[3].seconds += t[0] * 1e-3;
        S.prof[3].launches += 1;
        S.prof[0].seconds += t[1] * 1e-3;
        S.prof[0].launches += 1;
        S.prof[1].seconds += t[2] * 1e-3;
        S.prof[1].launches += 1;
        S.prof[2].seconds += t[3] * 1e-3;
        S.prof[2].launches += 1;
        if (h.hist_next >= h.hist_total && cnt_in[0] == 0 && cnt_in[1] == 0) break;
        if (h.flags & ERR_QUEUE) break;
        long long dthr = drain_threshold(e);
        if (dthr > 0 && h.hist_next >= h.hist_total && cnt_in[0] + cnt_in[1] <= dthr) {
            cudaEventRecord(ev[0], e->stream);
            launch_drain(e, oph, (long long)cnt_in[0] + cnt_in[1], tallies, (uint32_t)(seed >> 32), true);
            cudaEventRecord(ev[1], e->stream);
            if ((rc = cuda_check(e, cudaEventSynchronize(ev[1]), "drain"))) break;
            float td = 0;
            cudaEventElapsedTime(&td, ev[0], ev[1]);
            double row2[6] = {0.0, (double)cnt_in[0], (double)cnt_in[1], 0.0, 0.0, (double)td};
            S.trace.insert(S.trace.end(), row2, row2 + 6);
            S.prof[2].seconds += td * 1e-3;
            S.prof[2].launches += 1;
            cudaMemcpy(&h, S.ctl_d, sizeof(Ctl), cudaMemcpyDeviceToHost);
            double ds[5] = {(double)td, (double)cnt_in[0] + cnt_in[1], (double)h.drain_max_events,
                            (double)h.drain_max_chain, (double)h.drain_max_steps};
            std::copy(ds, ds + 5, S.drain_stats);
            break;
        }
        if (cycles > 200000) {
            rc = set_err(e, OMC_E_DEVICE, "event transport did not drain");
            break;
        }
    }
    for (auto &x : ev) cudaEventDestroy(x);
    return rc;
}

template <typename R>
int event_run_beam(omc_engine *e, const omc_beam *b, long nper, int nbatch, uint64_t seed, double *sum, double *sum2,
                   double *src_energy, KernelStats &ks) {
    if (sizeof(R) == 8 && e->d32.d.nsplit > 1)
        return set_err(e, OMC_E_RANGE, "the FP64 event form has no photon splitting (nsplit > 1)");
    int rc = event_prepare_t<R>(e);
    if (!rc) rc = event_interact_queue_t<R>(e);
    if (rc) return rc;
    EventStateT<R> &S = *state_of<R>(e);
    long nvox = e->ph.nvox();
    DBuf &tal = e->run_tal, &cdf = e->run_cdf32;
    if ((rc = tal.reserve((size_t)nbatch * nvox * 8))) return set_err(e, rc, "batch tallies allocation failed");
    cudaMemsetAsync(tal.p, 0, (size_t)nbatch * nvox * 8, e->stream);
    int ncdf = b->energy.n;
    BeamSrc<R> src = beam_setup<R>(e, b);
    if (ncdf > 0) {
        std::vector<R> c(b->energy.cdf1, b->energy.cdf1 + ncdf);
        c.insert(c.end(), b->energy.cdf2, b->energy.cdf2 + ncdf);
        if ((rc = cdf.reserve(c.size() * sizeof(R)))) return set_err(e, rc, "alloc");
        cudaMemcpyAsync(cdf.p, c.data(), c.size() * sizeof(R), cudaMemcpyHostToDevice, e->stream);
        src.cdf1 = cdf.as<R>();
        src.cdf2 = cdf.as<R>() + ncdf;
    }
    Ctl c0{};
    c0.hist_total = (long long)nper * nbatch;
    cudaMemcpyAsync(S.ctl_d, &c0, sizeof(Ctl), cudaMemcpyHostToDevice, e->stream);
    long long target = std::min<long long>((long long)S.cap / 2, S.inflight);

    if (e->opt.profile && sizeof(R) == 4) {
        Ctl h{};
        long cycles = 0;
        cudaEvent_t t0, t1;
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, e->stream);
        if constexpr (sizeof(R) == 4) rc = run_profiled(e, src, tal.as<double>(), nper, seed, target, h, cycles);
        for (int ib = 0; ib < nbatch && rc == OMC_OK; ib++)
            rc = fold(e, tal.as<double>() + (size_t)ib * nvox, sum, sum2, nvox, 1.0);
        cudaEventRecord(t1, e->stream);
        cudaEventSynchronize(t1);
        float ms = 0;
        cudaEventElapsedTime(&ms, t0, t1);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        ks.seconds = ms * 1e-3;
        ks.launches = cycles * (e->d32.d.defer_interact ? 5 : 4) + nbatch + (drain_threshold(e) > 0 ? 1 : 0);
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
    launch_cycle<R>(e, 0, src, tal.as<double>(), nper, seed, target);
    launch_cycle<R>(e, 1, src, tal.as<double>(), nper, seed, target);
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
    const long long dthr = drain_threshold_t<R>(e);
    int drains = 0;
    for (;;) {
        for (int k = 0; k < per_check; k++) cudaGraphLaunch(exec, e->stream);
        graphs += per_check;
        cudaMemcpyAsync(&h, S.ctl_d, sizeof(Ctl), cudaMemcpyDeviceToHost, e->stream);
        if ((rc = cuda_check(e, cudaStreamSynchronize(e->stream), "event transport"))) break;
        // a graph ends with a B -> A cycle: its outputs are queues A
        if (h.hist_next >= h.hist_total && h.cnt[0] == 0 && h.cnt[1] == 0 && h.cnt_hi[0] == 0 &&
            h.cnt_hi[1] == 0)
            break;
        if (h.flags & ERR_QUEUE) break;
        if (dthr > 0 && h.hist_next >= h.hist_total) {
            // every history is in: drain once few particles are left,
            // checking after every graph until then
            long long left = (long long)std::min(h.cnt[0] + h.cnt_hi[0], S.cap) +
                             std::min(h.cnt[1] + h.cnt_hi[1], S.cap);
            if (left <= dthr) {
                launch_drain<R>(e, 0, left, tal.as<double>(), (uint32_t)(seed >> 32));
                drains = 1;
                if ((rc = cuda_check(e, cudaStreamSynchronize(e->stream), "drain"))) break;
                cudaMemcpy(&h, S.ctl_d, sizeof(Ctl), cudaMemcpyDeviceToHost);
                break;
            }
            per_check = 1;
            continue;
        }
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
    ks.launches = graphs * (e->d32.d.defer_interact ? 10 : 8) + nbatch + drains;
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
template int event_run_beam<float>(omc_engine *, const omc_beam *, long, int, uint64_t, double *, double *, double *,
                                   KernelStats &);
template int event_run_beam<double>(omc_engine *, const omc_beam *, long, int, uint64_t, double *, double *, double *,
                                    KernelStats &);

// ============================================================== serving
// Inclusive prefix sum over the block (blockDim.x a multiple of 32, at most
// 1024) of one value per thread.
template <typename T>
__device__ __forceinline__ T block_inclusive_scan(T v, T *warp_tot) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) warp_tot[wid] = v;
    __syncthreads();
    if (wid == 0) {
        T w = lane < nw ? warp_tot[lane] : T(0);
        for (int o = 1; o < 32; o <<= 1) {
            T t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < nw) warp_tot[lane] = w;
    }
    __syncthreads();
    if (wid > 0) v += warp_tot[wid - 1];
    __syncthreads();
    return v;
}

// Histories to inject this cycle across the admitted requests, first come
// first served, keeping `target` particles in flight.  One block of
// SERVE_MAX threads, one per position in the admission order: request k
// takes min(its remaining histories, room left after requests 0..k-1),
// found by a prefix sum of the remaining histories.
__global__ void __launch_bounds__(SERVE_MAX) k_serve_plan(ServeDev *sd, Ctl *ctl, int iph, int iel, PlanCfg c) {
    __shared__ long long s_room;
    __shared__ long long warp_ll[SERVE_MAX / 32];
    __shared__ int warp_i[SERVE_MAX / 32];
    const int cap = c.cap;
    if (threadIdx.x == 0) {
        long long np, ne;
        plan_queues(ctl, iph, iel, cap, np, ne);
        long long room = (c.target - (np * c.pweight + ne)) / c.pweight;
        long long qroom = (long long)cap - (np > ne ? np : ne);
        if (room > qroom) room = qroom;
        s_room = room;
        plan_budget(ctl, ne, c);
    }
    __syncthreads();
    const long long room = s_room;
    const int k = threadIdx.x;
    int slot = -1;
    long long rem = 0, next = 0;
    if (k < sd->norder) {
        slot = sd->order[k];
        const ServeReq &r = sd->req[slot];
        if (r.kind >= 0 && r.nhist > r.next) {
            rem = r.nhist - r.next;
            next = r.next;
        }
    }
    const long long before = block_inclusive_scan(rem, warp_ll) - rem;
    long long take = room - before;
    take = take < 0 ? 0 : (take > rem ? rem : take);
    const int planned = take > 0;
    const int pos = block_inclusive_scan(planned, warp_i) - planned;
    if (planned) {
        // every request before this one got all it asked for: `before` is
        // the injections planned ahead of it
        sd->plan_slot[pos] = slot;
        sd->plan_first[pos] = next;
        sd->plan_cum[pos] = (int)before;
        sd->req[slot].next = next + take;
    }
    // the last thread sees the totals
    if (k == blockDim.x - 1) {
        const long long total_rem = before + rem;
        const long long total = total_rem < room ? total_rem : (room > 0 ? room : 0);
        const int nplan = pos + planned;
        sd->plan_cum[nplan] = (int)total;
        sd->nplan = nplan;
        sd->inject_total = (int)total;
    }
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
        SrcEnv<float> g;
        g.rng.init(key, seedw);
        float ein;
        Part<float> p = r.kind == 0 ? beam_primary(D, sd->beam[s], g, ein) : beamlet_primary(D, sd->bl[s], r.bixel, g, ein);
        int slot = s * nbmax + (int)(local / r.nper);
        int ip = warp_append(qP, p.iq == 0, false, active, flags);
        int ie = warp_append(qE, p.iq != 0, ctl->esplit > 0.f && p.e > ctl->esplit, active, flags);
        if (ip >= 0) qstore(qP, ip, p, slot, (uint32_t)key, (uint32_t)(key >> 32), g.rng.position());
        if (ie >= 0) qstore(qE, ie, p, slot, (uint32_t)key, (uint32_t)(key >> 32), g.rng.position());
        add_live(sd->live, nbmax, slot, (ip >= 0) + (ie >= 0), active);
    }
    unsigned active = __activemask();
    report_flags(ctl, flags, active);
}

void serve_launch_cycle(omc_engine *e, int in, ServeDev *sd, double *tallies, int nbmax, long long target) {
    EventState &S = *e->ev;
    int iph = in == 0 ? 0 : 2, iel = iph + 1;
    int oph = in == 0 ? 2 : 0, oel = oph + 1;
    const uint32_t seedw = SERVE_SEEDW;
    k_serve_plan<<<1, SERVE_MAX, 0, e->stream>>>(sd, S.ctl_d, iph, iel, plan_cfg(e, target));
    k_serve_source<<<S.grid, S.block, 0, e->stream>>>(e->d32.d, sd, S.q[iph], S.q[iel], S.ctl_d, nbmax, seedw);
    launch_transport(e, iph, iel, oph, oel, tallies, seedw, sd, nbmax, nullptr);
}

// A serving cycle launched on its own with an event around each kernel
// (engines created with options.profile): the per-kernel device time is
// added to the engine's profile; the transport counters are those the
// control block has accumulated since the server was created.
int serve_profiled_cycle(omc_engine *e, int in, ServeDev *sd, double *tallies, int nbmax, long long target) {
    EventState &S = *e->ev;
    int iph = in == 0 ? 0 : 2, iel = iph + 1;
    int oph = in == 0 ? 2 : 0, oel = oph + 1;
    const uint32_t seedw = SERVE_SEEDW;
    cudaEvent_t ev[5];
    for (auto &x : ev) cudaEventCreate(&x);
    cudaEventRecord(ev[0], e->stream);
    k_serve_plan<<<1, SERVE_MAX, 0, e->stream>>>(sd, S.ctl_d, iph, iel, plan_cfg(e, target));
    cudaEventRecord(ev[1], e->stream);
    k_serve_source<<<S.grid, S.block, 0, e->stream>>>(e->d32.d, sd, S.q[iph], S.q[iel], S.ctl_d, nbmax, seedw);
    cudaEventRecord(ev[2], e->stream);
    launch_transport(e, iph, iel, oph, oel, tallies, seedw, sd, nbmax, ev);
    cudaEventRecord(ev[4], e->stream);
    int rc = cuda_check(e, cudaEventSynchronize(ev[4]), "profiled serving cycle");
    if (!rc) {
        float t[4];
        for (int k = 0; k < 4; k++) cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]);
        const int map[4] = {3, 0, 1, 2};   // plan, source, photon, electron (+ interactions)
        for (int k = 0; k < 4; k++) {
            S.prof[map[k]].seconds += t[k] * 1e-3;
            S.prof[map[k]].launches += 1;
        }
        Ctl h{};
        cudaMemcpy(&h, S.ctl_d, sizeof(Ctl), cudaMemcpyDeviceToHost);
        for (int k = 0; k < 2; k++) {
            KernelProfile &P = S.prof[1 + k];
            P.particles = (double)h.st_events[k];
            P.steps = (double)h.st_steps[k];
            P.cross = (double)h.st_cross[k];
            P.dep = (double)h.st_dep[k];
            P.atom = (double)h.st_atom[k];
        }
    }
    for (auto &x : ev) cudaEventDestroy(x);
    return rc;
}

void serve_profile_reset(omc_engine *e) {
    for (auto &p : e->ev->prof) p = KernelProfile();
}

// The drain in serving: the particles left in queues A (where a graph of
// two cycles leaves them) run to the end on the serving streams; then the
// queues are emptied and every request's live count is zero.
void serve_drain(omc_engine *e, ServeDev *sd, long long left, double *tallies) {
    EventState &S = *e->ev;
    launch_drain(e, 0, left, tallies, SERVE_SEEDW);
    cudaMemsetAsync(sd->live, 0, sizeof(sd->live), e->stream);
    cudaMemsetAsync(S.ctl_d->cnt, 0, 2 * sizeof(int), e->stream);
    cudaMemsetAsync(S.ctl_d->cnt_hi, 0, 2 * sizeof(int), e->stream);
}

}  // namespace omc
