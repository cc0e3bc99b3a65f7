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
// Stack of the kernels used when photons are split: each split photon
// leaves up to about nsplit charged particles below its survivor, so the
// depth grows by about nsplit per photon generation (nsplit <= 64).
constexpr int SPLIT_STACK = 256;
// Transport steps (photon voxel steps + electron CH steps) one history may
// take before it is stopped with ERR_LOOP; typical histories take < 1e3.
constexpr long HISTORY_BUDGET = 2000000;

template <typename Rng>
struct PlainEnv {
    Rng rng;
    double *endep;       // per-voxel energy tally of the batch (index ir-1)
    Part<double> *st;    // the history's stack
    int cap;             // its capacity
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
        if (slot >= cap) {
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
    // the split photon's survivor is moved below its charged products
    static constexpr bool kRefOrder = false;
};

// Stack of the replay kernel (global memory, one per history): splitting
// in the reference's stack order leaves about nsplit/2 charged particles
// below each generation's surviving photon.
constexpr int REPLAY_STACK = 4096;

// photon() with photon splitting (ompmc.c:1867-2139, nsplit > 1) for the
// photon on top of the stack (slot np); returns the new top slot.  The
// photon is split into nsplit sub-photons of weight wt/nsplit whose
// interaction sites are stratified along its ray: sub-photon k travels
// -ln(eta_k) - sum of the previous ones' mean free paths from the previous
// site, with eta_k = 1 - (r + k)/nsplit.  Every sub-photon's charged
// products are kept; the scattered photon of one sub-photon, drawn at the
// start, survives with the full weight and the others' are removed.  Once
// the loop ends a photon on top of the stack is split again at once.
template <typename Env>
__device__ int photon_split(const DevData<double> &D, Env &g, Part<double> *st, int np) {
    const int ns = D.nsplit;
    double eig = st[np].e;
    int irl = st[np].ir;
    if (eig <= pcut_of(D, irl) || st[np].wt == 0.0) {
        g.deposit(irl, st[np].wt * eig);
        return np - 1;
    }
    double gle = log(eig);
    for (int resplit = 0;; resplit++) {
        if (resplit > 100000) {
            g.err(ERR_LOOP);
            return -1;
        }
        double rnno = g.uni();
        rnno /= (double)ns;
        const double d_eta = 1.0 / (double)ns;
        double eta_prime = 1.0 - rnno + d_eta;
        Part<double> save = st[np];
        const double wtsave = save.wt / (double)ns;
        const int s0 = np;
        np -= 1;
        rnno = g.uni();
        const int isurv = (int)(rnno * ns);
        double dpmfp_old = 0.0;
        for (int isplit = 0; isplit < ns; isplit++) {
            eta_prime -= d_eta;
            if (eta_prime <= 0.0) break;
            double dpmfp = -log(eta_prime) - dpmfp_old;
            dpmfp_old += dpmfp;
            np += 1;
            if (np >= g.cap) {
                g.err(ERR_STACK);
                return -1;
            }
            Part<double> q = save;
            q.wt = wtsave;
            q.iq = 0;
            int imed, lgle;
            double cohfac;
            if (!photon_walk(D, g, q, gle, dpmfp, imed, lgle, cohfac)) {
                np -= 1;     // discarded: the rest of the ray lies beyond it
                break;
            }
            save.x = q.x; save.y = q.y; save.z = q.z;
            save.ir = q.ir;
            rnno = g.uni();
            if (rnno <= 1.0 - cohfac) {
                if (isplit != isurv) {
                    np -= 1;
                } else {
                    q.wt *= ns;
                    rayleigh(D, g, q, imed, gle, lgle);
                    st[np] = q;
                }
                continue;
            }
            g.top = np;
            g.nchild = 0;
            photon_interact(D, g, q, eig, gle, imed, lgle);
            st[np] = q;
            int ip = np;
            np += g.nchild;
            // the non-surviving sub-photons' scattered photons leave the
            // stack: the top entry moves into the freed slot (all products
            // of the interaction share its position and region)
            do {
                if (st[ip].iq == 0) {
                    if (isplit != isurv) {
                        if (ip < np) {
                            st[ip].e = st[np].e; st[ip].iq = st[np].iq;
                            st[ip].u = st[np].u; st[ip].v = st[np].v; st[ip].w = st[np].w;
                            st[ip].wt = st[np].wt;
                        }
                        np -= 1;
                    } else {
                        st[ip].wt *= ns;
                        ip += 1;
                    }
                } else {
                    ip += 1;
                }
            } while (ip <= np);
        }
        if (!Env::kRefOrder) {
            // transport this photon's charged products before its surviving
            // photon, so that the stack does not grow with every photon
            // generation (the reference leaves the survivor among them); the
            // order of independent particles does not change the expected
            // dose
            for (int k = s0 + 1; k <= np; k++)
                if (st[k].iq == 0) {
                    Part<double> t = st[s0];
                    st[s0] = st[k];
                    st[k] = t;
                    break;
                }
        }
        if (np < 0 || st[np].iq != 0) return np;
        eig = st[np].e;
        irl = st[np].ir;
        if (eig <= pcut_of(D, irl)) {
            g.deposit(irl, st[np].wt * eig);
            return np - 1;
        }
        gle = log(eig);
    }
}

// shower() (ompmc.c:5454-5465) on a local stack.
template <typename Env>
__device__ void shower(const DevData<double> &D, Env &g, Part<double> *st) {
    int np = 0;
    long steps = 0;
    g.work = 0;
    while (np >= 0) {
        if (st[np].iq == 0 && D.nsplit > 1) {
            np = photon_split(D, g, st, np);
        } else {
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
        }
        if (++steps > 100000) {
            g.err(ERR_LOOP);
            break;
        }
        if (g.flags & (ERR_RNG | ERR_LOOP)) break;
    }
}

template <int CAP>
__global__ void k_plain_beam(DevData<double> D, BeamSrc<double> S, double *endep, uint64_t seed, long hist0, long n,
                             double *src_energy, unsigned *errw) {
    PlainEnv<Philox<double>> g;
    Part<double> st[CAP];
    g.endep = endep;
    g.st = st;
    g.cap = CAP;
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

template <int CAP>
__global__ void k_plain_beamlet(DevData<double> D, BeamletSrc<double> S, int ib, double *endep, uint64_t seed,
                                long hist0, long n, unsigned *errw) {
    PlainEnv<Philox<double>> g;
    Part<double> st[CAP];
    g.endep = endep;
    g.st = st;
    g.cap = CAP;
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
    static constexpr bool kRefOrder = true;
    ScriptRng rng;
    Part<double> *st;
    int cap;
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
        if (slot >= cap) {
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
                         int dep_cap, int *dep_ir, double *dep_e, int *ndep, long *nused, unsigned *flags,
                         Part<double> *stacks) {
    int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nhist) return;
    ReplayEnv g;
    Part<double> *st = stacks + (long)h * REPLAY_STACK;
    g.cap = REPLAY_STACK;
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

// Histories per launch of the plain form: about four seconds of FP64
// transport, so that a large batch is a sequence of bounded launches.  A
// history's random stream depends on its index only, so the split does not
// change the result.
static const long PLAIN_CHUNK = 1L << 22;

int plain_beam_batch(omc_engine *e, const BeamSrc<double> &S, double *work, uint64_t seed, long hist0, long n,
                     double *src_energy, int block, long *launches) {
    const bool split = e->d64.d.nsplit > 1;
    for (long c0 = 0; c0 < n; c0 += PLAIN_CHUNK) {
        if (launches) ++*launches;
        long c = std::min(PLAIN_CHUNK, n - c0);
        if (split)
            k_plain_beam<SPLIT_STACK><<<grid_for(e, c, block), block, 0, e->stream>>>(
                e->d64.d, S, work, seed, hist0 + c0, c, src_energy, e->errword.as<unsigned>());
        else
            k_plain_beam<PLAIN_STACK><<<grid_for(e, c, block), block, 0, e->stream>>>(
                e->d64.d, S, work, seed, hist0 + c0, c, src_energy, e->errword.as<unsigned>());
        int rc = cuda_check(e, cudaGetLastError(), "k_plain_beam launch");
        if (rc) return rc;
    }
    return OMC_OK;
}

int plain_beamlet_batch(omc_engine *e, const BeamletSrc<double> &S, int ib, double *work, uint64_t seed, long hist0,
                        long n, int block) {
    if (e->d64.d.nsplit > 1)
        k_plain_beamlet<SPLIT_STACK><<<grid_for(e, n, block), block, 0, e->stream>>>(e->d64.d, S, ib, work, seed,
                                                                                      hist0, n,
                                                                                      e->errword.as<unsigned>());
    else
        k_plain_beamlet<PLAIN_STACK><<<grid_for(e, n, block), block, 0, e->stream>>>(e->d64.d, S, ib, work, seed,
                                                                                      hist0, n,
                                                                                      e->errword.as<unsigned>());
    return cuda_check(e, cudaGetLastError(), "k_plain_beamlet launch");
}

int plain_trace(omc_engine *e, const double *rays_d, int nrays, int cap, double *ustep, int *irnew, int *idisc,
                int *ncalls, double *hn) {
    k_trace<<<(nrays + 127) / 128, 128, 0, e->stream>>>(e->d64.d, rays_d, nrays, cap, ustep, irnew, idisc, ncalls,
                                                        hn);
    return cuda_check(e, cudaGetLastError(), "k_trace launch");
}

size_t plain_replay_stack_bytes(int nhist) { return (size_t)nhist * REPLAY_STACK * sizeof(Part<double>); }

int plain_replay(omc_engine *e, const double *prim, int nhist, const double *rn, const long *rn_off, int dep_cap,
                 int *dep_ir, double *dep_e, int *ndep, long *nused, unsigned *flags, void *stacks) {
    k_replay<<<(nhist + 63) / 64, 64, 0, e->stream>>>(e->d64.d, prim, nhist, rn, rn_off, dep_cap, dep_ir, dep_e, ndep,
                                                      nused, flags, (Part<double> *)stacks);
    return cuda_check(e, cudaGetLastError(), "k_replay launch");
}

// ------------------------------------------ sampler known-answer hooks
// One interaction sampler (or one msdist step) per case on a scripted
// uniform stream, with the FP64 physics of this translation unit (no
// contracted multiply-adds, like the x86 reference).  The particle itself
// is output 0, what the sampler pushes follows.
struct KatEnv {
    static constexpr bool kRefOrder = true;
    ScriptRng rng;
    Part<double> out[KAT_MAXOUT];
    int nout;
    unsigned flags;
    long work;
    double edep;
    __device__ bool tick() { return ++work < HISTORY_BUDGET; }
    __device__ double uni() { return rng.uni(); }
    __device__ void deposit(int, double e) { edep += e; }
    __device__ bool push(const Part<double> &q) {
        if (nout + 1 >= KAT_MAXOUT) {
            flags |= ERR_STACK;
            return false;
        }
        out[++nout] = q;
        return true;
    }
    __device__ void err(unsigned f) { flags |= f; }
    __device__ void cross() {}
    __device__ bool tstep_take() const { return true; }
};

__global__ void k_kat(DevData<double> D, int which, const double *q, const double *extra, int n, const double *rn,
                      const long *rn_off, double *out, int *nout, long *used, unsigned *flags) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const double *a = q + 11 * (long)c;
    Part<double> p{a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], (int)a[8], (int)a[9]};
    KatEnv g;
    unsigned fl = 0;
    g.rng = ScriptRng{rn + rn_off[c], rn_off[c + 1] - rn_off[c], 0, &fl};
    g.nout = 0;
    g.flags = 0;
    g.work = 0;
    g.edep = 0.0;
    double *o = out + (long)c * KAT_MAXOUT * 11;
    for (int k = 0; k < KAT_MAXOUT * 11; k++) o[k] = 0.0;
    const int imed = p.ir > 0 ? D.med[p.ir] : 0;
    if (which == KAT_MSDIST) {
        double xf, yf, zf, uf, vf, wf;
        double ustep = msdist(D, g, p, imed, p.iq, D.rhof[p.ir], extra[2 * c], extra[2 * c + 1], p.e - D_RM, xf, yf, zf,
                              uf, vf, wf);
        double r[7] = {ustep, xf, yf, zf, uf, vf, wf};
        for (int k = 0; k < 7; k++) o[k] = r[k];
        nout[c] = 1;
    } else {
        const double gle = log(p.e);
        switch (which) {
        case 0: compton(D, g, p); break;
        case 1: photo(D, g, p); break;
        case 2: pair(D, g, p, imed); break;
        case 3: rayleigh(D, g, p, imed, gle, lidx(D.ms[imed].ge1, D.ms[imed].ge0, gle)); break;
        case 4: moller(D, g, p); break;
        case 5: bhabha(D, g, p); break;
        case 6: brems(D, g, p); break;
        case 7: annih(D, g, p); break;
        case 8: rannih(D, g, p); break;
        default: g.flags |= ERR_LOOP; break;
        }
        g.out[0] = p;
        for (int i = 0; i <= g.nout; i++) {
            const Part<double> &t = g.out[i];
            double r[10] = {t.x, t.y, t.z, t.u, t.v, t.w, t.e, t.wt, (double)t.ir, (double)t.iq};
            for (int k = 0; k < 10; k++) o[11 * i + k] = r[k];
        }
        nout[c] = g.nout + 1;
    }
    used[c] = g.rng.pos;
    flags[c] = g.flags | fl;
}

int plain_kat(omc_engine *e, int which, const double *q, const double *extra, int n, const double *rn,
              const long *rn_off, double *out, int *nout, long *used, unsigned *flags) {
    k_kat<<<(n + 63) / 64, 64, 0, e->stream>>>(e->d64.d, which, q, extra, n, rn, rn_off, out, nout, used, flags);
    return cuda_check(e, cudaGetLastError(), "k_kat launch");
}

}  // namespace omc
