// Plain form: FP64, history-based, one thread per history with a local LIFO
// particle stack — the direct GPU analogue of ompMC's OpenMP loop
// (omc_dosxyz.c:1252-1259: initHistory(); shower();).  Also the trajectory
// and geometry validation kernels, which need FP64 and the reference's
// operation order.  This file is compiled with -fmad=false so that no
// multiply-add is contracted (the x86 reference has none).
#include <cstdio>

#include "omc_engine.h"
#include "omc_rng.cuh"
#include "omc_source.cuh"

namespace omc {

constexpr int PLAIN_STACK = 48;
// Transport steps (photon voxel steps + electron CH steps) one history may
// take before it is stopped with ERR_LOOP; typical histories take < 1e3.
constexpr long HISTORY_BUDGET = 2000000;

template <typename Rng>
struct PlainEnv {
    Rng rng;
    double *endep;       // per-voxel energy tally of the batch (index ir-1)
    Part<double> *st;    // the history's stack
    int top;             // slot of the particle being processed
    int nchild;          // particles pushed above it
    unsigned flags;
    long work;
    __device__ bool tick() { return ++work < HISTORY_BUDGET; }
    __device__ double uni() { return rng.uni(); }
    __device__ void deposit(int ir, double e) {
        if (ir > 0 && e != 0.0) atomicAdd(&endep[ir - 1], e);
    }
    __device__ bool push(const Part<double> &q) {
        int slot = top + 1 + nchild;
        if (slot >= PLAIN_STACK) {
            flags |= ERR_STACK;
            return false;
        }
        st[slot] = q;
        nchild++;
        return true;
    }
    __device__ void err(unsigned f) { flags |= f; }
    __device__ void cross() {}
    __device__ bool tstep_take() const { return true; }
};

// shower() (ompmc.c:5454-5465) on a local stack.
template <typename Env>
__device__ void shower(const DevData<double> &D, Env &g, Part<double> *st) {
    int np = 0;
    long steps = 0;
    g.work = 0;
    while (np >= 0) {
        Part<double> p = st[np];
        g.top = np;
        g.nchild = 0;
        int alive = (p.iq == 0) ? (int)photon_step(D, g, p) : electron_step(D, g, p);
        if (alive) {
            st[np] = p;
            np += g.nchild;
        } else {
            for (int k = 0; k < g.nchild; k++) st[np + k] = st[np + 1 + k];
            np += g.nchild - 1;
        }
        if (++steps > 100000) {
            g.err(ERR_LOOP);
            break;
        }
        if (g.flags & (ERR_RNG | ERR_LOOP)) break;
    }
}

__global__ void k_plain_beam(DevData<double> D, BeamSrc<double> S, double *endep, uint64_t seed, long hist0, long n,
                             double *src_energy, unsigned *errw) {
    PlainEnv<Philox<double>> g;
    Part<double> st[PLAIN_STACK];
    g.endep = endep;
    g.st = st;
    g.flags = 0;
    double esum = 0;
    for (long h = blockIdx.x * (long)blockDim.x + threadIdx.x; h < n; h += (long)gridDim.x * blockDim.x) {
        g.rng.init(mix64(seed ^ (uint64_t)(hist0 + h) * 0x9E3779B97F4A7C15ull), (uint32_t)(seed >> 32));
        double ein;
        st[0] = beam_primary(D, S, g, ein);
        esum += ein;
        shower(D, g, st);
    }
    if (g.flags) atomicOr(errw, g.flags);
    if (src_energy) atomicAdd(src_energy, esum);
}

__global__ void k_plain_beamlet(DevData<double> D, BeamletSrc<double> S, int ib, double *endep, uint64_t seed,
                                long hist0, long n, unsigned *errw) {
    PlainEnv<Philox<double>> g;
    Part<double> st[PLAIN_STACK];
    g.endep = endep;
    g.st = st;
    g.flags = 0;
    for (long h = blockIdx.x * (long)blockDim.x + threadIdx.x; h < n; h += (long)gridDim.x * blockDim.x) {
        g.rng.init(mix64(seed ^ ((uint64_t)ib << 40) ^ (uint64_t)(hist0 + h) * 0x9E3779B97F4A7C15ull),
                   (uint32_t)(seed >> 32));
        double ein;
        st[0] = beamlet_primary(D, S, ib, g, ein);
        shower(D, g, st);
    }
    if (g.flags) atomicOr(errw, g.flags);
}

// ------------------------------------------------------------ validation
__global__ void k_trace(DevData<double> D, const double *rays, int nrays, int cap, double *ustep, int *irnew,
                        int *idisc, int *ncalls, double *hn) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrays) return;
    Part<double> p;
    p.x = rays[7 * r]; p.y = rays[7 * r + 1]; p.z = rays[7 * r + 2];
    p.u = rays[7 * r + 3]; p.v = rays[7 * r + 4]; p.w = rays[7 * r + 5];
    p.ir = (int)rays[7 * r + 6];
    p.e = 1; p.wt = 1; p.iq = 0;
    if (hn) hn[r] = hownear(D, p);
    int n = 0;
    while (n < cap) {
        int id = 0, irn = p.ir;
        double us = 1.0E8;
        howfar(D, p, id, irn, us);
        ustep[(long)r * cap + n] = us;
        irnew[(long)r * cap + n] = irn;
        idisc[(long)r * cap + n] = id;
        n++;
        if (id > 0) break;
        p.x += us * p.u;
        p.y += us * p.v;
        p.z += us * p.w;
        p.ir = irn;
    }
    ncalls[r] = n;
}

// Uniforms read from a recorded stream.
struct ScriptRng {
    const double *rn;
    long n, pos;
    unsigned *flags;
    uint32_t spare = 0x2545F491u;
    // Past the end of the stream: flag it and continue on a small xorshift
    // so that rejection loops still terminate; the history is then stopped.
    __device__ double uni() {
        if (pos < n) return rn[pos++];
        *flags |= ERR_RNG;
        pos++;
        spare ^= spare << 13;
        spare ^= spare >> 17;
        spare ^= spare << 5;
        return u01d(spare);
    }
};

struct ReplayEnv {
    ScriptRng rng;
    Part<double> *st;
    int top, nchild;
    unsigned flags;
    int *dep_ir;
    double *dep_e;
    int dep_cap, ndep;
    long work;
    __device__ bool tick() { return ++work < HISTORY_BUDGET; }
    __device__ double uni() { return rng.uni(); }
    __device__ void deposit(int ir, double e) {
        if (ndep < dep_cap) {
            dep_ir[ndep] = ir;
            dep_e[ndep] = e;
        } else {
            flags |= ERR_LOG;
        }
        ndep++;
    }
    __device__ bool push(const Part<double> &q) {
        int slot = top + 1 + nchild;
        if (slot >= PLAIN_STACK) {
            flags |= ERR_STACK;
            return false;
        }
        st[slot] = q;
        nchild++;
        return true;
    }
    __device__ void err(unsigned f) { flags |= f; }
    __device__ void cross() {}
    __device__ bool tstep_take() const { return true; }
};

__global__ void k_replay(DevData<double> D, const double *prim, int nhist, const double *rn, const long *rn_off,
                         int dep_cap, int *dep_ir, double *dep_e, int *ndep, long *nused, unsigned *flags) {
    int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nhist) return;
    ReplayEnv g;
    Part<double> st[PLAIN_STACK];
    g.flags = 0;
    g.rng.rn = rn + rn_off[h];
    g.rng.n = rn_off[h + 1] - rn_off[h];
    g.rng.pos = 0;
    g.rng.flags = &g.flags;
    g.st = st;
    g.dep_ir = dep_ir + (long)h * dep_cap;
    g.dep_e = dep_e + (long)h * dep_cap;
    g.dep_cap = dep_cap;
    g.ndep = 0;
    const double *q = prim + 11 * (long)h;
    Part<double> &p = st[0];
    p.x = q[0]; p.y = q[1]; p.z = q[2];
    p.u = q[3]; p.v = q[4]; p.w = q[5];
    p.e = q[6]; p.wt = q[7]; p.ir = (int)q[8]; p.iq = (int)q[9];
    shower(D, g, st);
    ndep[h] = g.ndep;
    nused[h] = g.rng.pos;
    flags[h] = g.flags;
}

// ------------------------------------------------------------ launchers
static int grid_for(omc_engine *e, long n, int block) {
    long g = (n + block - 1) / block;
    long cap = (long)e->sm_count * 16;
    if (g > cap) g = cap;
    return (int)(g < 1 ? 1 : g);
}

int plain_beam_batch(omc_engine *e, const BeamSrc<double> &S, double *work, uint64_t seed, long hist0, long n,
                     double *src_energy, int block) {
    k_plain_beam<<<grid_for(e, n, block), block, 0, e->stream>>>(e->d64.d, S, work, seed, hist0, n, src_energy,
                                                                  e->errword.as<unsigned>());
    return cuda_check(e, cudaGetLastError(), "k_plain_beam launch");
}

int plain_beamlet_batch(omc_engine *e, const BeamletSrc<double> &S, int ib, double *work, uint64_t seed, long hist0,
                        long n, int block) {
    k_plain_beamlet<<<grid_for(e, n, block), block, 0, e->stream>>>(e->d64.d, S, ib, work, seed, hist0, n,
                                                                     e->errword.as<unsigned>());
    return cuda_check(e, cudaGetLastError(), "k_plain_beamlet launch");
}

int plain_trace(omc_engine *e, const double *rays_d, int nrays, int cap, double *ustep, int *irnew, int *idisc,
                int *ncalls, double *hn) {
    k_trace<<<(nrays + 127) / 128, 128, 0, e->stream>>>(e->d64.d, rays_d, nrays, cap, ustep, irnew, idisc, ncalls,
                                                        hn);
    return cuda_check(e, cudaGetLastError(), "k_trace launch");
}

int plain_replay(omc_engine *e, const double *prim, int nhist, const double *rn, const long *rn_off, int dep_cap,
                 int *dep_ir, double *dep_e, int *ndep, long *nused, unsigned *flags) {
    k_replay<<<(nhist + 63) / 64, 64, 0, e->stream>>>(e->d64.d, prim, nhist, rn, rn_off, dep_cap, dep_ir, dep_e, ndep,
                                                      nused, flags);
    return cuda_check(e, cudaGetLastError(), "k_replay launch");
}

}  // namespace omc
