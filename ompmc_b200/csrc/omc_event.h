// Event-based FP32 transport form (omc_event.cu).
#pragma once
#include <vector>
#include "omc_engine.h"

namespace omc {

// Particle queue in device memory: four arrays of 16-, 16-, 16- and 4-byte
// elements (FP32 form), so a warp moves a particle's 52 bytes with three
// 128-bit and one 32-bit coalesced access each way: pos = (x, y, z, u),
// dir = (v, w, e, wt), id = (ir, tag, k0, k1), ctr.  The FP64 event form
// keeps pos and dir in double (84 bytes per particle).  `tag` packs the charge (iq+1, 2 bits)
// and the tally slot (upper bits); k0/k1 are the particle's Philox stream
// key and ctr its stream position (numbers drawn).  Entries fill from both
// ends: `count` entries from index 0 up and `count_hi` entries from index
// cap-1 down (electron queues put particles above the regroup energy at
// the top, so that warps see particles of one kind).
template <typename R>
struct QVec;
template <>
struct QVec<float> {
    using T = float4;
};
template <>
struct QVec<double> {
    using T = double4;   // two 128-bit accesses
};

template <typename R>
struct QueueT {
    typename QVec<R>::T *pos, *dir;
    uint4 *id;
    uint32_t *ctr;
    // photon splitting state (photon queues of engines with nsplit > 1,
    // else null): -1 for a photon not yet split, else (next sub-photon << 16)
    // | surviving sub-photon; and the ray's stratification offset
    int *sp;
    float *sr;
    int *count;      // device counter of entries from the bottom
    int *count_hi;   // device counter of entries from the top
    int cap;
};
using Queue = QueueT<float>;

// Cycle control block in device memory.
struct Ctl {
    int cnt[4];               // photon A, electron A, photon B, electron B (from the bottom)
    int cnt_hi[4];            // the same queues, entries from the top
    int cnt_int, cnt_int_hi;  // electrons waiting for their discrete interaction (this cycle)
    long long hist_next;      // next history to inject
    long long hist_total;     // histories requested
    int inject;               // histories injected this cycle
    int inject_base_lo;       // unused padding
    long long hist_base;      // first history of this cycle's injection
    unsigned flags;           // DevErr bits
    int pad;
    double src_energy;        // sum of primary kinetic energies
    int tsteps;               // this cycle's electron budget (tstep-loop iterations per event)
    float esplit;             // regroup energy (total, MeV): electrons above it go to the top
    int fetch[3];             // work counters of the photon, electron and interaction kernels
    int pad3;
    // counters per transport kernel (0 photon, 1 electron)
    unsigned long long st_events[2], st_steps[2], st_cross[2], st_dep[2], st_atom[2];
    // drain: the largest sub-history one thread ran (events, events of the
    // particle it started from, transport steps)
    int drain_max_events, drain_max_chain, drain_max_steps, drain_pad;
};

// Per-kernel profile of the last run made with options.profile = 1.
struct KernelProfile {
    double launches = 0, seconds = 0, particles = 0, steps = 0, cross = 0, dep = 0, atom = 0;
};

// Per-cycle planning parameters passed to the planner kernels.
struct PlanCfg {
    long long target;         // particles kept in flight
    int cap;                  // queue capacity
    int lanes;                // resident threads of the transport kernels
    int boost;                // largest budget multiplier as the queues drain (1 = fixed)
    int tsteps;               // base electron budget (tstep-loop iterations)
    float esplit;             // regroup energy of the electron queues (total, MeV; 0 = one group)
    int pweight;              // in-flight weight of a queued photon: nsplit (each makes up to
                              // nsplit charged particles), 1 without splitting
};

template <typename R>
struct EventStateT {
    bool ready = false;
    int cap = 0;              // per queue
    DBuf buf[4];              // photon A, electron A, photon B, electron B (13 arrays each)
    DBuf split_buf[2];        // splitting state of the photon queues (nsplit > 1)
    DBuf int_buf;             // electrons at their discrete interaction (defer_interact)
    QueueT<R> qi;
    QueueT<R> q[4];
    DBuf ctl;
    Ctl *ctl_d = nullptr;
    int block = 256;
    int grid = 0;             // source kernels
    int grid_p = 0, grid_e = 0, grid_i = 0;  // transport kernels: one wave of resident blocks
    int lanes = 0;            // resident threads of the electron kernel
    int drain_lanes = 0;      // resident threads of the drain kernel
    int boost = 32;           // budget multiplier limit in the drain tail
    int tsteps = 2;           // electron tstep iterations per event launch
    double esplit = 0;        // regroup energy of the electron queues (total, MeV)
    long long inflight = 0;   // particles kept in flight by the injector
    KernelProfile prof[4];    // 0 source, 1 photon, 2 electron, 3 plan+reset
    // profiled runs: per cycle {histories injected, photons in, electrons in,
    // source ms, photon ms, electron ms}
    std::vector<double> trace;
    // profiled runs: the drain's ms, particles, and largest sub-history
    // (events, events of its first particle, transport steps); zeros if none
    double drain_stats[5] = {0, 0, 0, 0, 0};
    // second stream of the captured cycles: the photon kernel runs there,
    // beside the electron kernels of its cycle (fork/join events)
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    ~EventStateT() {
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        if (side) cudaStreamDestroy(side);
    }
};
using EventState = EventStateT<float>;

// ------------------------------------------------------------ serving
constexpr int SERVE_MAX = 256;  // request slots resident on the device
constexpr uint32_t SERVE_SEEDW = 0x5e7e5eedu;  // seed word of the serving streams

// One admitted request: its histories are injected from `next` on; kind -1
// marks a free slot.
struct ServeReq {
    int kind;            // -1 free, 0 beam, 1 beamlet
    int bixel;
    long long nhist, next, nper;
    unsigned long long seed;
};

// Device-resident request table and the per-cycle injection plan.
struct ServeDev {
    ServeReq req[SERVE_MAX];
    BeamSrc<float> beam[SERVE_MAX];
    BeamletSrc<float> bl[SERVE_MAX];
    int live[SERVE_MAX];       // particles of the request in the queues
    int order[SERVE_MAX];      // active slots in admission order
    int norder;
    int nplan;
    int inject_total;
    int pad;
    int plan_slot[SERVE_MAX];
    long long plan_first[SERVE_MAX];
    int plan_cum[SERVE_MAX + 1];
};

int event_prepare(omc_engine *e);
int event_interact_queue(omc_engine *e);
// One serving cycle with input buffers `in` (0 = A, 1 = B); tally slot of a
// particle = request slot * nbmax + batch.
void serve_launch_cycle(omc_engine *e, int in, ServeDev *sd, double *tallies, int nbmax, long long target);
void serve_drain(omc_engine *e, ServeDev *sd, long long left, double *tallies);
int serve_profiled_cycle(omc_engine *e, int in, ServeDev *sd, double *tallies, int nbmax, long long target);
void serve_profile_reset(omc_engine *e);
// Particles left at or below which a run whose histories are all injected
// switches from transport cycles to the drain kernel (0: never).
long long drain_threshold(const omc_engine *e);
PlanCfg plan_cfg(const omc_engine *e, long long target);
int event_set_params(omc_engine *e, int tsteps, int boost, long long inflight, int block, double split_kinetic);

// The event form's dose run in precision R (float: FP32 transport; double:
// the FP64 event form, OMC_EVENT_FP64).
template <typename R>
int event_run_beam(omc_engine *e, const omc_beam *b, long nper, int nbatch, uint64_t seed, double *sum, double *sum2,
                   double *src_energy, KernelStats &ks);
void event_release(omc_engine *e);
template <typename R>
BeamSrc<R> beam_setup(const omc_engine *e, const omc_beam *b);
int fold(omc_engine *e, double *work, double *sum, double *sum2, long n, double scale);
}  // namespace omc
