// Device data model shared by every transport kernel.
//
// Tables are interleaved per energy bin so one bin is one or two vector
// loads: a piecewise-linear table entry is a pair {slope a1, intercept a0},
// evaluated as a1*lnE + a0 (ompMC pwlfEval, src/ompmc.c:204-212).
#pragma once
#include <cstdint>

namespace omc {

#ifndef OMC_HD
#define OMC_HD __host__ __device__ __forceinline__
#endif
#ifndef OMC_COLD
// Interaction samplers and other code that runs at most once per event:
// one out-of-line copy keeps the transport kernels small enough for the
// instruction caches.
#define OMC_COLD __host__ __device__ __noinline__
#endif
#ifndef OMC_OUTLINE
// Large routines called from several sites of the electron step (one copy
// instead of one per call site, for the same reason).
#define OMC_OUTLINE __host__ __device__ __noinline__
#endif

constexpr int D_MXGE = 2000;
constexpr int D_MXEKE = 500;
constexpr int D_MXRAYFF = 100;
constexpr int D_MXMED = 9;
constexpr int D_NE1 = 32;       // spin energies
constexpr int D_NQ1 = 16;       // spin q1 bins
constexpr int D_NU1 = 32;       // spin u bins
constexpr int D_NMS = 64 * 8 * 32;

template <typename R>
struct alignas(2 * sizeof(R)) PL {
    R a1, a0;
};

// Photon bin: mean free path, Rayleigh correction, branching ratios.
template <typename R>
struct PhBin {
    PL<R> gmfp, cohe, gbr1, gbr2;
};

// Electron bin for one charge (0 = e-, 1 = e+).  `range` is the CSDA range
// from the first grid energy to the bin's lower edge, `earr` that edge.
template <typename R>
struct ElBin {
    PL<R> sig, dedx, tmxs, eta, blcce, q1c, q2c, br1, br2;
    R range, earr;
};

template <typename R>
struct MsE {
    R u, f, w;
    int i;
};

// Per-medium scalars.
template <typename R>
struct MedS {
    R ge0, ge1, eke0, eke1;
    R blcc, xcc, sige[2];
    R te, thmoll, ap, ae;
    R delcm, zbrang, bpar0, bpar1;
    R pcut, ecut;        // transport cut-offs in this medium
    R dl1[8], dl2[8], dl3[8], dl4[8], dl5[8], dl6[8];
    int ismono[2];
    int meke;
    int pad;
};

template <typename R>
struct Rayl {
    R xgrid[D_MXRAYFF], fcum[D_MXRAYFF], b[D_MXRAYFF], c[D_MXRAYFF];
    int ia[D_MXRAYFF];
};

// Division of a non-negative 32-bit integer n < 2^31 by a run-time
// constant d >= 1 with a multiply-high, an add and a shift (Granlund and
// Montgomery, "Division by invariant integers using multiplication", PLDI
// 1994): with s = ceil(log2 d) and M = floor(2^(32+s) / d) + 1 < 2^33,
// n / d = floor(n M / 2^(32+s)) exactly for every n < 2^32; M = 2^32 + m
// with m < 2^32 gives n / d = (mulhi(n, m) + n) >> s, and the sum stays
// below 2^32 for n < 2^31.  The GPU has no integer divide instruction.
struct FastDiv {
    uint32_t d, m, s;
    static FastDiv make(uint32_t d) {
        FastDiv f{d, 0u, 0u};
        if (d > (1u << 31)) {
            // every n < 2^31 is below d: m = 0, s = 31 gives n >> 31 = 0
            f.s = 31;
            return f;
        }
        while ((1ull << f.s) < d) f.s++;
        f.m = (uint32_t)(((1ull << (32 + f.s)) / d + 1) - (1ull << 32));
        return f;
    }
    __host__ __device__ __forceinline__ uint32_t div(uint32_t n) const {
#ifdef __CUDA_ARCH__
        const uint32_t hi = __umulhi(n, m);
#else
        const uint32_t hi = (uint32_t)(((uint64_t)n * m) >> 32);
#endif
        return (hi + n) >> s;
    }
};

template <typename R>
struct DevData {
    int nmed;
    int nx, ny, nz;
    FastDiv div_nx, div_nxy;         // n / nx and n / (nx*ny) for region indices
    const R *xb, *yb, *zb;          // voxel boundaries
    const int8_t *med;               // [nvox+1] medium index per region, -1 = vacuum / outside
    const R *rhof;                   // [nvox+1] density / PEGS density
    const MedS<R> *ms;               // [nmed]
    const PhBin<R> *ph;              // [nmed*MXGE]
    const PL<R> *pmax;               // [nmed*MXGE]
    const Rayl<R> *ray;              // [nmed]
    const ElBin<R> *el;              // [(nmed*2)*MXEKE]: (imed*2+qel)*MXEKE + bin
    const MsE<R> *msurf;             // [NMS]
    const R *spin;                   // [nmed][2][32][16][32]
    R b2spin_min, dbeta2i, espml, dleneri, dqq1i, dllambi, dqmsi;
    int ref_compat;                  // reproduce reference quirks (default 1)
    int nsplit;                      // photon splitting factor (1 = off)
    int chsteps;                     // electrons: condensed-history steps after which the
                                     // distance to the next discrete interaction is re-drawn
                                     // (0 = the reference's restart after every step)
    int defer_interact;              // electrons: leave discrete interactions to a separate
                                     // kernel (event form) instead of sampling them in place
    // photons: delta (Woodcock) tracking on a uniform voxel grid (event form)
    int woodcock;                    // 1: photons walk by delta tracking, not voxel by voxel
    int uniform;                     // the grid is uniform on all three axes
    R gx0, gy0, gz0;                 // lower corner of the grid
    R gx1, gy1, gz1;                 // upper corner
    R gidx, gidy, gidz;              // 1 / voxel size per axis
    R rhomax[D_MXMED];               // largest density ratio of each medium in the phantom
};

// Beam source of the dosxyz ucode (omc_dosxyz.c:337-632, :964-1068).
template <typename R>
struct BeamSrc {
    int charge;
    int spectrum;                    // 0 mono, 1 spectrum
    R energy;
    const R *cdf1, *cdf2;            // inverse CDF [deltak]
    R deltak;
    R ssd, xinl, yinl, xsize, ysize;
    int ixinl, iyinl;
};

// Beamlet source of the matRad ucode (omc_matrad.c:1177-1413).
template <typename R>
struct BeamletSrc {
    int charge, spectrum, gaussian;
    R energy, gauss_width;
    const R *cdf1, *cdf2;
    R deltak;
    // per beamlet
    const int *ibeam;
    const R *src;     // [nbeams*3] source position per beam
    const R *corner;  // [nbixels*3]
    const R *side1;   // [nbixels*3]
    const R *side2;   // [nbixels*3]
};

// Device error flags (or-ed into a word the host reads after each run).
enum DevErr : unsigned {
    ERR_STACK = 1u,          // history stack overflow; particle dropped
    ERR_LOOP = 2u,           // step-count guard tripped; particle dropped
    ERR_QUEUE = 4u,          // queue overflow; particle dropped
    ERR_RNG = 8u,            // scripted random stream exhausted
    ERR_LOG = 16u,           // deposit log full
    ERR_LAMBDA = 32u,        // BCA lambda_max <= 0; particle dropped (as the reference)
    ERR_NAN = 64u,           // non-finite state; particle dropped
};

}  // namespace omc
