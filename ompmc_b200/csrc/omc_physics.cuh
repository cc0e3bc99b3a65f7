// Coupled photon/electron class II condensed-history transport on the GPU.
//
// A from-scratch restatement of the EGSnrc algorithm as ompMC runs it
// (src/ompmc.c); every function cites the reference lines whose results it
// reproduces.  Random numbers are drawn in the reference's order, one call
// of the environment's uni() per setRandom() call, so that the FP64
// instantiation replayed on a recorded reference stream follows the same
// trajectory (the parity tests rely on it).
//
// Templates:
//   R    float (event-based FP32 transport) or double (plain FP64 form)
//   Env  the environment: R uni(); void deposit(int ir, R e);
//        bool push(const Part<R>&); void err(unsigned); void cross() (a
//        voxel boundary was crossed; counting only); bool tstep_take()
//        (false once the caller's budget of tstep-loop iterations is spent:
//        electron_step then returns the particle for a later call, which
//        resumes it exactly); bool tick() (false
//        once the history's transport-step budget is spent; every loop
//        that could run away is bounded by it or by a local guard)
//
// Reference quirks reproduced when D.ref_compat != 0 (the default) are
// marked "quirk"; each is listed in the design notes.
#pragma once
#include <cmath>

#include "omc_device.cuh"

namespace omc {

constexpr double D_RM = 0.5109989461;

template <typename R>
struct Part {
    R x, y, z, u, v, w, e, wt;
    int ir, iq;
};

// ------------------------------------------------------------ math shims
// FP32 transport uses the hardware log2/exp2 based intrinsics (a few
// instructions each instead of an inlined library routine at each of some
// forty call sites); their errors (about 2^-21 absolute near 1) are far below
// the FP32 transport's own rounding.
OMC_HD double m_log(double x) { return log(x); }
OMC_HD double m_exp(double x) { return exp(x); }
#ifdef __CUDA_ARCH__
OMC_HD float m_log(float x) { return __logf(x); }
OMC_HD float m_exp(float x) { return __expf(x); }
#else
OMC_HD float m_log(float x) { return logf(x); }
OMC_HD float m_exp(float x) { return expf(x); }
#endif
OMC_HD double m_sqrt(double x) { return sqrt(x); }
OMC_HD float m_sqrt(float x) { return sqrtf(x); }
OMC_HD double m_sin(double x) { return sin(x); }
OMC_HD float m_sin(float x) { return sinf(x); }
OMC_HD double m_cos(double x) { return cos(x); }
OMC_HD float m_cos(float x) { return cosf(x); }
OMC_HD double m_pow(double x, double y) { return pow(x, y); }
OMC_HD float m_pow(float x, float y) { return powf(x, y); }
template <typename R> OMC_HD R m_max(R a, R b) { return a > b ? a : (b == b ? b : a); }
template <typename R> OMC_HD R m_min(R a, R b) { return a < b ? a : (b == b ? b : a); }
template <typename R> OMC_HD R sq(R x) { return x * x; }
template <typename R> OMC_HD bool m_abs_lt(R a, R b) { return (a < R(0) ? -a : a) < b; }

// FP32 transport renormalises a direction wherever it is rotated, so that
// rounding drift never accumulates and the trajectory does not depend on
// where events are cut; the FP64 form is left untouched (its trajectories
// stay bit-identical to the reference's).
OMC_HD void renorm_dir(double &, double &, double &) {}
OMC_HD void renorm_dir(float &u, float &v, float &w) {
    float n2 = u * u + v * v + w * w;
    if (n2 > 0.f && fabsf(n2 - 1.f) > 1e-6f) {
#ifdef __CUDA_ARCH__
        float r = rsqrtf(n2);
#else
        float r = 1.0f / sqrtf(n2);
#endif
        u *= r; v *= r; w *= r;
    }
}

template <typename R>
OMC_HD R pwl(const PL<R> &p, R x) { return x * p.a1 + p.a0; }

// Interval of a log-energy grid, C indexing: (int)(c1*lnE + c0) - 1
// (pwlfInterval, ompmc.c:204-207).
template <typename R>
OMC_HD int lidx(R c1, R c0, R le) { return (int)(le * c1 + c0) - 1; }

template <typename R>
OMC_HD R ecut_of(const DevData<R> &D, int ir) {
    int m = D.med[ir];
    return m >= 0 ? D.ms[m].ecut : R(0);
}
template <typename R>
OMC_HD R pcut_of(const DevData<R> &D, int ir) {
    int m = D.med[ir];
    return m >= 0 ? D.ms[m].pcut : R(0);
}

template <typename R>
OMC_HD const ElBin<R> &ebin(const DevData<R> &D, int imed, int qel, int l) {
    int meke = D.ms[imed].meke;
    l = l < 0 ? 0 : (l >= meke ? meke - 1 : l);
    return D.el[(imed * 2 + qel) * D_MXEKE + l];
}
template <typename R>
OMC_HD const PhBin<R> &pbin(const DevData<R> &D, int imed, int l) {
    l = l < 0 ? 0 : (l >= D_MXGE ? D_MXGE - 1 : l);
    return D.ph[imed * D_MXGE + l];
}

// ------------------------------------------------------------- geometry
// Column, row and plane of region irl (1-based, x fastest): the
// reference's (irl-1) % nx, / (nx*ny) and / nx, by exact multiply-high
// divisions.
template <typename R>
OMC_HD void voxel_ijk(const DevData<R> &D, int irl, int &irx, int &iry, int &irz) {
    const uint32_t n = (uint32_t)(irl - 1);
    const uint32_t k = D.div_nxy.div(n);
    const uint32_t r = n - k * D.div_nxy.d;
    const uint32_t j = D.div_nx.div(r);
    irx = (int)(r - j * D.div_nx.d);
    iry = (int)j;
    irz = (int)k;
}

// Distance to the next voxel plane along the direction, checked in the
// order z, x, y; the new region is the neighbour across that plane or 0
// (outside); a particle already outside is discarded
// (howfar, omc_dosxyz.c:187-297).
template <typename R>
OMC_HD void howfar(const DevData<R> &D, const Part<R> &p, int &idisc, int &irnew, R &ustep) {
    int irl = p.ir;
    if (irl == 0) {
        idisc = 1;
        return;
    }
    int imax = D.nx, ijmax = D.nx * D.ny;
    int irx, iry, irz;
    voxel_ijk(D, irl, irx, iry, irz);
    R dist;
    if (p.w > R(0)) {
        dist = (D.zb[irz + 1] - p.z) / p.w;
        if (dist < ustep) { ustep = dist; irnew = (irz != D.nz - 1) ? irl + ijmax : 0; }
    } else if (p.w < R(0)) {
        dist = -(p.z - D.zb[irz]) / p.w;
        if (dist < ustep) { ustep = dist; irnew = (irz != 0) ? irl - ijmax : 0; }
    }
    if (p.u > R(0)) {
        dist = (D.xb[irx + 1] - p.x) / p.u;
        if (dist < ustep) { ustep = dist; irnew = (irx != D.nx - 1) ? irl + 1 : 0; }
    } else if (p.u < R(0)) {
        dist = -(p.x - D.xb[irx]) / p.u;
        if (dist < ustep) { ustep = dist; irnew = (irx != 0) ? irl - 1 : 0; }
    }
    if (p.v > R(0)) {
        dist = (D.yb[iry + 1] - p.y) / p.v;
        if (dist < ustep) { ustep = dist; irnew = (iry != D.ny - 1) ? irl + imax : 0; }
    } else if (p.v < R(0)) {
        dist = -(p.y - D.yb[iry]) / p.v;
        if (dist < ustep) { ustep = dist; irnew = (iry != 0) ? irl - imax : 0; }
    }
}

// Isotropic distance to the nearest face of the current voxel
// (hownear, omc_dosxyz.c:299-334).
template <typename R>
OMC_HD R hownear(const DevData<R> &D, const Part<R> &p) {
    int irl = p.ir;
    if (irl == 0) return R(0);
    int irx, iry, irz;
    voxel_ijk(D, irl, irx, iry, irz);
    R t = R(1.0E10);
    t = m_min(t, D.xb[irx + 1] - p.x);
    t = m_min(t, p.x - D.xb[irx]);
    t = m_min(t, D.yb[iry + 1] - p.y);
    t = m_min(t, p.y - D.yb[iry]);
    t = m_min(t, D.zb[irz + 1] - p.z);
    t = m_min(t, p.z - D.zb[irz]);
    return t;
}

// ------------------------------------------------------------ rotations
// Azimuth by rejection in the unit half disc (selectAzimuthalAngle,
// ompmc.c:102-125).
template <typename R, typename Env>
OMC_HD void azimuth(Env &g, R &cphi, R &sphi) {
    R x, x2, y, y2, r2;
    int guard = 0;
    do {
        x = g.uni();
        x = R(2) * x - R(1);
        x2 = x * x;
        y = g.uni();
        y2 = y * y;
        r2 = x2 + y2;
        if (++guard > 1000) { g.err(ERR_LOOP); x2 = R(1); y2 = R(0); x = R(1); y = R(0); r2 = R(1); break; }
    } while (r2 > R(1));
    r2 = R(1) / r2;
    cphi = (x2 - y2) * r2;
    sphi = R(2) * x * y * r2;
}

template <typename R>
struct Uphi {
    R A, B, C, cphi, sphi;
};

template <typename R>
OMC_HD void rotate_into(R A, R B, R C, R costhe, R sinthe, R cphi, R sphi, R &u, R &v, R &w) {
    R sinps2 = A * A + B * B;
    if (sinps2 < R(1.0E-20)) {
        u = sinthe * cphi;
        v = sinthe * sphi;
        w = C * costhe;
    } else {
        R sinpsi = m_sqrt(sinps2);
        R us = sinthe * cphi, vs = sinthe * sphi;
        R sindel = B / sinpsi, cosdel = A / sinpsi;
        u = C * cosdel * us - sindel * vs + A * costhe;
        v = C * sindel * us + cosdel * vs + B * costhe;
        w = -sinpsi * us + C * costhe;
    }
}

// New direction of the current particle; keeps the old direction and the
// azimuth for a correlated partner (uphi21, ompmc.c:128-165).
template <typename R, typename Env>
OMC_HD void uphi21(Env &g, Part<R> &p, Uphi<R> &h, R costhe, R sinthe) {
    azimuth(g, h.cphi, h.sphi);
    h.A = p.u; h.B = p.v; h.C = p.w;
    rotate_into(h.A, h.B, h.C, costhe, sinthe, h.cphi, h.sphi, p.u, p.v, p.w);
    renorm_dir(p.u, p.v, p.w);
}

// Partner particle: position, region and weight of p, direction rotated
// from p's direction before uphi21 (uphi32, ompmc.c:167-202).
template <typename R>
OMC_HD Part<R> uphi32(const Part<R> &p, const Uphi<R> &h, R costhe, R sinthe) {
    Part<R> q = p;
    rotate_into(h.A, h.B, h.C, costhe, sinthe, h.cphi, h.sphi, q.u, q.v, q.w);
    renorm_dir(q.u, q.v, q.w);
    return q;
}

// ------------------------------------------------------ photon samplers
// Rayleigh: form-factor sampling with Thomson rejection
// (rayleigh, ompmc.c:1120-1163).  quirk: the bin index is
// `(int)rnno0*dwi` == 0 and the form-factor tables of medium 0 are used
// for every medium.
template <typename R, typename Env>
OMC_HD void rayleigh_body(const DevData<R> &D, Env &g, Part<R> &p, int imed, R gle, int lgle) {
    R eig = p.e;
    R pmax = pwl(D.pmax[imed * D_MXGE + (lgle < 0 ? 0 : (lgle > D_MXGE - 1 ? D_MXGE - 1 : lgle))], gle);
    R xmax = R(80.65506856998) * eig;
    const Rayl<R> &ry = D.ray[D.ref_compat ? 0 : imed];
    R rnno0, rnno1, xv, costhe, csqthe;
    int guard = 0;
    do {
        rnno1 = g.uni();
        do {
            if (++guard > 100000) { g.err(ERR_LOOP); xv = R(0); break; }
            rnno0 = g.uni();
            rnno0 *= pmax;
            int ibin = D.ref_compat ? 0 : (int)(rnno0 * R(99));
            if (ibin > 98) ibin = 98;
            int ib = ry.ia[ibin] - 1;
            if (ry.ia[ibin + 1] - 1 > ib)
                while (ib < D_MXRAYFF - 2 && rnno0 >= ry.fcum[ib + 1]) ib++;
            rnno0 = (rnno0 - ry.fcum[ib]) * ry.c[ib];
            xv = ry.xgrid[ib] * m_exp(m_log(R(1) + rnno0) * ry.b[ib]);
        } while (xv >= xmax);
        xv /= eig;
        costhe = R(1) - R(0.000307444456) * (xv * xv);
        csqthe = costhe * costhe;
    } while (R(2) * rnno1 >= (R(1) + csqthe));
    R sinthe = m_sqrt(R(1) - csqthe);
    Uphi<R> h;
    uphi21(g, p, h, costhe, sinthe);
}

// Out-of-line copy (the plain form, the split photons and the electron
// kernels call it by reference).
template <typename R, typename Env>
OMC_COLD void rayleigh(const DevData<R> &D, Env &g, Part<R> &p, int imed, R gle, int lgle) {
    rayleigh_body(D, g, p, imed, gle, lgle);
}

// Pair rejection function in xi (PIRS-0287 eq. 4; ompmc.c:1436-1445).
template <typename R>
OMC_HD R pair_rej(R zbrang, R xi, R esedei, R eseder, R tteig) {
    return R(2) + R(3) * (esedei + eseder) -
           R(4) * (esedei + eseder + R(1) - R(4) * sq(xi - R(0.5))) *
               (R(1) + R(0.25) * m_log(sq((R(1) + eseder) * (R(1) + esedei) / (R(2) * tteig)) + zbrang * sq(xi)));
}

// Pair production: uniform split below 2.1 MeV, Bethe-Heitler (with
// Coulomb correction above 50 MeV) screening rejection otherwise; angles
// from the Motz-Olsen-Koch leading term (pair, ompmc.c:1447-1685).
// p becomes particle 1 and particle 2 is pushed.  quirk: the angle loop
// accepts as soon as theta < pi.
template <typename R, typename Env>
OMC_HD void pair_body(const DevData<R> &D, Env &g, Part<R> &p, int imed) {
    const MedS<R> &M = D.ms[imed];
    const R RMr = R(D_RM);
    R eig = p.e, ese1, ese2;
    int iq1, iq2;
    if (eig <= R(2.1)) {
        R r0 = g.uni(), r1 = g.uni();
        ese2 = RMr + R(0.5) * r0 * (eig - R(2) * RMr);
        ese1 = eig - ese2;
        if (r1 < R(0.5)) { iq1 = -1; iq2 = 1; } else { iq1 = 1; iq2 = -1; }
    } else {
        int l, l1;
        R Amax, Bmax, aux, delta;
        if (eig < R(50)) {
            l = 4; l1 = 5;
            delta = R(4) * M.delcm / eig;
            if (delta < R(1)) {
                Amax = M.dl1[l] + delta * (M.dl2[l] + delta * M.dl3[l]);
                Bmax = M.dl1[l1] + delta * (M.dl2[l1] + delta * M.dl3[l1]);
            } else {
                aux = m_log(delta + M.dl6[l]);
                Amax = M.dl4[l] + M.dl5[l] * aux;
                Bmax = M.dl4[l1] + M.dl5[l1] * aux;
            }
            aux = R(1) - R(2) * RMr / eig;
            aux = aux * aux;
            aux *= Amax / R(3);
            aux /= (Bmax + aux);
        } else {
            l = 6;
            Amax = M.dl1[l];
            Bmax = M.dl1[l + 1];
            aux = M.bpar1 * (R(1) - M.bpar0 * RMr / eig);
        }
        R eavail = eig - R(2) * RMr, rejf, rejmax, r4;
        int guard = 0;
        do {
            R r0 = g.uni(), r1 = g.uni();
            r4 = g.uni();
            R br;
            if (r0 > aux) {
                br = R(0.5) * r1;
                rejmax = Bmax;
                l1 = l + 1;
            } else {
                R r2 = g.uni(), r3 = g.uni();
                br = R(0.5) * (R(1) - m_max(m_max(r1, r2), r3));
                rejmax = Amax;
                l1 = l;
            }
            ese2 = br * eavail + RMr;
            ese1 = eig - ese2;
            delta = (eig * M.delcm) / (ese2 * ese1);
            if (delta < R(1))
                rejf = M.dl1[l1] + delta * (M.dl2[l1] + delta * M.dl3[l1]);
            else
                rejf = M.dl4[l1] + M.dl5[l1] * m_log(delta + M.dl6[l1]);
            if (++guard > 100000) { g.err(ERR_LOOP); break; }
        } while (r4 * rejmax > rejf);
        ese1 = eig - ese2;
        r4 = g.uni();
        if (r4 < R(0.5)) { iq1 = -1; iq2 = 1; } else { iq1 = 1; iq2 = -1; }
    }
    p.e = ese1;
    Part<R> q = p;
    q.e = ese2;
    Uphi<R> h;
    for (int j = 0; j < 2; j++) {
        R ese = j == 0 ? ese1 : ese2;
        R tteig = eig / RMr, ttese = ese / RMr;
        R esedei = ttese / (tteig - ttese), eseder = R(1) / esedei;
        R ximin = R(1) / (R(1) + sq(R(M_PI) * ttese));
        R rejmin = pair_rej(M.zbrang, ximin, esedei, eseder, tteig);
        R ya = sq(R(2) / tteig);
        R xitry = m_max(R(0.01), m_max(ximin, m_min(R(0.5), m_sqrt(ya / M.zbrang))));
        R galpha = R(1) + R(0.25) * m_log(ya + M.zbrang * xitry * xitry);
        R gbeta = R(0.5) * M.zbrang * xitry / (ya + M.zbrang * xitry * xitry);
        galpha -= gbeta * (xitry - R(0.5));
        R ximid = galpha / (R(3) * gbeta);
        if (galpha >= R(0)) ximid = R(0.5) - ximid + m_sqrt(ximid * ximid + R(0.25));
        else ximid = R(0.5) - ximid - m_sqrt(ximid * ximid + R(0.25));
        ximid = m_max(R(0.01), m_max(ximin, m_min(R(0.5), ximid)));
        R rejmid = pair_rej(M.zbrang, ximid, esedei, eseder, tteig);
        R rejtop = R(1) * m_max(rejmin, rejmid);
        R theta, rtest, rejfactor;
        int guard = 0;
        do {
            R xitst = g.uni();
            R rejtst = pair_rej(M.zbrang, xitst, esedei, eseder, tteig);
            rtest = g.uni();
            theta = m_sqrt(R(1) / xitst - R(1)) / ttese;
            rejfactor = rejtst / rejtop;
            if (++guard > 100000) { g.err(ERR_LOOP); break; }
        } while (D.ref_compat ? ((rtest > rejfactor) && (theta >= R(M_PI))) : ((rtest > rejfactor) || (theta >= R(M_PI))));
        R sinthe = m_sin(theta), costhe = m_cos(theta);
        if (j == 0) {
            uphi21(g, p, h, costhe, sinthe);
        } else {
            Part<R> r = uphi32(p, h, costhe, -sinthe);
            q.u = r.u; q.v = r.v; q.w = r.w;
        }
    }
    p.iq = iq1;
    q.iq = iq2;
    g.push(q);
}

// Out-of-line copy (the plain form, the split photons and the electron
// kernels call it by reference).
template <typename R, typename Env>
OMC_COLD void pair(const DevData<R> &D, Env &g, Part<R> &p, int imed) {
    pair_body(D, g, p, imed);
}

// Compton scattering off free electrons, Klein-Nishina (compton,
// ompmc.c:1688-1801).  p stays the scattered photon; the electron is pushed.
template <typename R, typename Env>
OMC_HD void compton_body(const DevData<R> &D, Env &g, Part<R> &p) {
    const R RMr = R(D_RM);
    R eig = p.e, ko = p.e / RMr;
    R broi = R(1) + R(2) * ko, bro = R(1) / broi;
    bool first = true;
    R sinthe = 0, br = 0, temp = 0, alph1 = 0, alph2 = 0, alpha = 0, rejmax = 0;
    int guard = 0;
    do {
        if (ko > R(2)) {
            if (first) {
                alph1 = m_log(broi);
                alph2 = ko * (broi + R(1)) * (bro * bro);
                alpha = alph1 + alph2;
            }
            R r1, r2, r3, aux, rejf3;
            do {
                r1 = g.uni();
                r2 = g.uni();
                if (r1 * alpha < alph1) br = m_exp(alph1 * r2) * bro;
                else br = m_sqrt(r2 * (broi * broi) + (R(1) - r2)) * bro;
                temp = (R(1) - br) / (ko * br);
                sinthe = m_max(R(0), temp * (R(2) - temp));
                aux = R(1) + br * br;
                rejf3 = aux - br * sinthe;
                r3 = g.uni();
                if (++guard > 100000) { g.err(ERR_LOOP); break; }
            } while (r3 * aux > rejf3);
        } else {
            if (first) rejmax = broi + bro;
            R r1, r2, rejf3;
            do {
                r1 = g.uni();
                r2 = g.uni();
                br = bro + (R(1) - bro) * r1;
                temp = (R(1) - br) / (ko * br);
                sinthe = m_max(R(0), temp * (R(2) - temp));
                rejf3 = R(1) + br * br - br * sinthe;
                if (++guard > 100000) { g.err(ERR_LOOP); break; }
            } while (r2 * br * rejmax > rejf3);
        }
        first = false;
        if (guard > 100000) break;
    } while ((br < bro) || (br > R(1)));
    R costhe = R(1) - temp;
    sinthe = m_sqrt(sinthe);
    R esg = br * eig, ese = eig - esg + RMr;
    p.e = esg;
    Uphi<R> h;
    uphi21(g, p, h, costhe, sinthe);
    R aux = R(1) + br * br - R(2) * br * costhe;
    if (aux > R(1.0E-8)) {
        costhe = (R(1) - br * costhe) / m_sqrt(aux);
        sinthe = (R(1) - costhe) * (R(1) + costhe);
        sinthe = sinthe > R(0) ? -m_sqrt(sinthe) : R(0);
    } else {
        costhe = R(0);
        sinthe = R(-1);
    }
    Part<R> q = uphi32(p, h, costhe, sinthe);
    q.e = ese;
    q.iq = -1;
    g.push(q);
}

// Out-of-line copy (the plain form, the split photons and the electron
// kernels call it by reference).
template <typename R, typename Env>
OMC_COLD void compton(const DevData<R> &D, Env &g, Part<R> &p) {
    compton_body(D, g, p);
}

// Photo-absorption: the photon becomes an electron with E + m, emitted
// along the Sauter distribution when above the region's cut-off
// (photo, ompmc.c:1804-1864).
template <typename R, typename Env>
OMC_HD void photo_body(const DevData<R> &D, Env &g, Part<R> &p) {
    const R RMr = R(D_RM);
    p.e += RMr;
    p.iq = -1;
    R eelec = p.e;
    if (eelec > ecut_of(D, p.ir)) {
        R beta = m_sqrt((eelec - RMr) * (eelec + RMr)) / eelec;
        R gamma = eelec / RMr;
        R alpha = R(0.5) * gamma - R(0.5) + R(1) / gamma;
        R ratio = beta / alpha;
        R costhe, sinth2, xi, rnpht2;
        int guard = 0;
        do {
            R rnpht = g.uni();
            rnpht = R(2) * rnpht - R(1);
            if (ratio <= R(0.2)) {
                R fkappa = rnpht + R(0.5) * ratio * (R(1) - rnpht) * (R(1) + rnpht);
                if (gamma < R(100)) {
                    costhe = (beta + fkappa) / (R(1) + beta * fkappa);
                } else if (fkappa > R(0)) {
                    costhe = R(1) - (R(1) - fkappa) * (gamma - R(3)) / (R(2) * (R(1) + fkappa) * m_pow(gamma - R(1), R(3)));
                } else {
                    costhe = (beta + fkappa) / (R(1) + beta * fkappa);
                }
                xi = (R(1) + beta * fkappa) * (gamma * gamma);
            } else {
                xi = (gamma * gamma) * (R(1) + alpha * (m_sqrt(R(1) + ratio * (R(2) * rnpht + ratio)) - R(1)));
                costhe = (R(1) - R(1) / xi) / beta;
            }
            sinth2 = m_max((R(1) - costhe) * (R(1) + costhe), R(0));
            rnpht2 = g.uni();
            if (++guard > 100000) { g.err(ERR_LOOP); break; }
        } while (rnpht2 > R(0.5) * (R(1) + gamma) * sinth2 * xi / gamma);
        R sinthe = m_sqrt(sinth2);
        Uphi<R> h;
        uphi21(g, p, h, costhe, sinthe);
    }
}

// Out-of-line copy (the plain form, the split photons and the electron
// kernels call it by reference).
template <typename R, typename Env>
OMC_COLD void photo(const DevData<R> &D, Env &g, Part<R> &p) {
    photo_body(D, g, p);
}

// Environments that declare kInlineSamplers = true (the out-of-line photon
// event of the event form) get the photon samplers inlined; every other
// caller uses their out-of-line copies.
template <typename Env, typename = void>
struct InlineSamplers {
    static constexpr bool value = false;
};
template <typename Env>
struct InlineSamplers<Env, decltype((void)Env::kInlineSamplers)> {
    static constexpr bool value = Env::kInlineSamplers;
};
template <typename R, typename Env>
OMC_HD void rayleigh_at(const DevData<R> &D, Env &g, Part<R> &p, int imed, R gle, int lgle) {
    if constexpr (InlineSamplers<Env>::value) rayleigh_body(D, g, p, imed, gle, lgle);
    else rayleigh(D, g, p, imed, gle, lgle);
}
template <typename R, typename Env>
OMC_HD void pair_at(const DevData<R> &D, Env &g, Part<R> &p, int imed) {
    if constexpr (InlineSamplers<Env>::value) pair_body(D, g, p, imed);
    else pair(D, g, p, imed);
}
template <typename R, typename Env>
OMC_HD void compton_at(const DevData<R> &D, Env &g, Part<R> &p) {
    if constexpr (InlineSamplers<Env>::value) compton_body(D, g, p);
    else compton(D, g, p);
}
template <typename R, typename Env>
OMC_HD void photo_at(const DevData<R> &D, Env &g, Part<R> &p) {
    if constexpr (InlineSamplers<Env>::value) photo_body(D, g, p);
    else photo(D, g, p);
}

// --------------------------------------------------------- photon step
// Voxel walk of a photon to its interaction site `dpmfp` mean free paths
// ahead (the transport loop of photon, ompmc.c:1957-2037).  Returns false
// when the photon leaves the geometry (or a guard trips); otherwise p is at
// the site and imed, lgle and cohfac are those of the site's medium.
template <typename R, typename Env>
OMC_HD bool photon_walk(const DevData<R> &D, Env &g, Part<R> &p, R gle, R dpmfp, int &imed, int &lgle, R &cohfac) {
    int irl = p.ir;
    int irold = irl;
    imed = D.med[irl];
    lgle = 0;
    cohfac = 0;
    R gmfp = 0;
    int guard = 0;
    for (;;) {
        R tstep;
        if (imed != -1) {
            const MedS<R> &M = D.ms[imed];
            lgle = lidx(M.ge1, M.ge0, gle);
            const PhBin<R> &b = pbin(D, imed, lgle);
            R gmfpr0 = pwl(b.gmfp, gle);
            gmfp = gmfpr0 / D.rhof[irl];
            cohfac = pwl(b.cohe, gle);
            gmfp *= cohfac;
            tstep = gmfp * dpmfp;
        } else {
            tstep = R(1.0E8);
        }
        int irnew = irl, idisc = 0;
        R ustep = tstep;
        howfar(D, p, idisc, irnew, ustep);
        p.x += ustep * p.u;
        p.y += ustep * p.v;
        p.z += ustep * p.w;
        if (idisc > 0) return false;
        if (imed != -1) dpmfp = m_max(R(0), dpmfp - ustep / gmfp);
        if (irnew != irold) {
            p.ir = irnew;
            irl = irnew;
            irold = irnew;
            imed = D.med[irl];
            g.cross();
        }
        if (imed != -1 && dpmfp <= R(1.0E-5)) return true;
        if (++guard > 100000 || !g.tick()) { g.err(ERR_LOOP); return false; }
    }
}

// The interaction at the end of a walk, after the Rayleigh draw came out
// against Rayleigh: pair, Compton or photo-absorption by the branching
// ratios of the site (ompmc.c:2060-2085).  p becomes the interaction's
// first product; a second one, if any, is pushed.
template <typename R, typename Env>
OMC_HD void photon_interact(const DevData<R> &D, Env &g, Part<R> &p, R eig, R gle, int imed, int lgle) {
    R rnno = g.uni();
    const PhBin<R> &b = pbin(D, imed, lgle);
    R gbr1 = pwl(b.gbr1, gle);
    if (rnno <= gbr1 && eig > R(2) * R(D_RM)) {
        pair_at(D, g, p, imed);
    } else {
        R gbr2 = pwl(b.gbr2, gle);
        if (rnno < gbr2) compton_at(D, g, p);
        else photo_at(D, g, p);
    }
}

// One call of photon(): cut-off check, number of mean free paths, voxel
// walk to the interaction site and the interaction (photon, ompmc.c:1867-2139
// with nsplit = 1).  Returns false when the photon is gone.
template <typename R, typename Env>
OMC_HD bool photon_step(const DevData<R> &D, Env &g, Part<R> &p) {
    R eig = p.e;
    int irl = p.ir;
    if (eig <= pcut_of(D, irl) || p.wt == R(0)) {
        g.deposit(irl, p.wt * eig);
        return false;
    }
    R gle = m_log(eig);
    // nsplit = 1: the mean-free-path draw and the survivor draw
    R rnno = g.uni();
    R eta_prime = (R(1) - rnno + R(1)) - R(1);
    (void)g.uni();
    R dpmfp = -m_log(eta_prime);
    int imed, lgle;
    R cohfac;
    if (!photon_walk(D, g, p, gle, dpmfp, imed, lgle, cohfac)) return false;
    rnno = g.uni();
    if (rnno <= R(1) - cohfac) {
        rayleigh_at(D, g, p, imed, gle, lgle);
        return true;
    }
    photon_interact(D, g, p, eig, gle, imed, lgle);
    return true;
}

// Photon event by delta (Woodcock) tracking, for uniform voxel grids (the
// event form; D.woodcock).  The same physics as photon_step: the distance
// to the next real interaction is exponential in the local attenuation
// mu(x) = rhof(x) / (gmfp(E) * cohfac(E)) of the voxel medium, sampled here
// against the largest attenuation mu_max of the phantom at this energy:
// tentative steps of -ln(xi)/mu_max, each accepted as a real interaction
// with probability mu(x)/mu_max (a standard, exact method; Woodcock et
// al. 1965).  A photon in a 0.25 cm grid then takes a few steps per event
// instead of one per voxel crossed.  The interaction itself is photon_step's.
template <typename R, typename Env>
OMC_HD bool photon_step_delta(const DevData<R> &D, Env &g, Part<R> &p) {
    R eig = p.e;
    if (eig <= pcut_of(D, p.ir) || p.wt == R(0)) {
        g.deposit(p.ir, p.wt * eig);
        return false;
    }
    R gle = m_log(eig);
    R mu_max = 0;
    for (int m = 0; m < D.nmed; m++) {
        const MedS<R> &M = D.ms[m];
        const PhBin<R> &b = pbin(D, m, lidx(M.ge1, M.ge0, gle));
        mu_max = m_max(mu_max, D.rhomax[m] / (pwl(b.gmfp, gle) * pwl(b.cohe, gle)));
    }
    if (!(mu_max > R(0))) return false;
    // distance to the grid's boundary along the direction
    R texit = R(1.0E30);
    if (p.u > R(0)) texit = m_min(texit, (D.gx1 - p.x) / p.u);
    else if (p.u < R(0)) texit = m_min(texit, (D.gx0 - p.x) / p.u);
    if (p.v > R(0)) texit = m_min(texit, (D.gy1 - p.y) / p.v);
    else if (p.v < R(0)) texit = m_min(texit, (D.gy0 - p.y) / p.v);
    if (p.w > R(0)) texit = m_min(texit, (D.gz1 - p.z) / p.w);
    else if (p.w < R(0)) texit = m_min(texit, (D.gz0 - p.z) / p.w);
    const R x0 = p.x, y0 = p.y, z0 = p.z;
    const R inv_mu = R(1) / mu_max;
    R t = 0;
    int imed = -1, lgle = 0;
    R cohfac = 0;
    for (int guard = 0;; guard++) {
        if (guard > 100000 || !g.tick()) {
            g.err(ERR_LOOP);
            return false;
        }
        t += -m_log(R(1) - g.uni()) * inv_mu;
        if (t >= texit) return false;   // leaves the phantom
        R x = x0 + t * p.u, y = y0 + t * p.v, z = z0 + t * p.w;
        int i = min(max((int)((x - D.gx0) * D.gidx), 0), D.nx - 1);
        int j = min(max((int)((y - D.gy0) * D.gidy), 0), D.ny - 1);
        int k = min(max((int)((z - D.gz0) * D.gidz), 0), D.nz - 1);
        int ir = 1 + i + D.nx * (j + D.ny * k);
        int m = D.med[ir];
        R r = g.uni();
        if (m < 0) continue;
        const MedS<R> &M = D.ms[m];
        int l = lidx(M.ge1, M.ge0, gle);
        const PhBin<R> &b = pbin(D, m, l);
        R coh = pwl(b.cohe, gle);
        R mu = D.rhof[ir] / (pwl(b.gmfp, gle) * coh);
        if (r * mu_max <= mu) {
            p.x = x; p.y = y; p.z = z;
            if (ir != p.ir) g.cross();
            p.ir = ir;
            imed = m;
            lgle = l;
            cohfac = coh;
            break;
        }
    }
    R rnno = g.uni();
    if (rnno <= R(1) - cohfac) {
        rayleigh_at(D, g, p, imed, gle, lgle);
        return true;
    }
    photon_interact(D, g, p, eig, gle, imed, lgle);
    return true;
}

// ------------------------------------------ the out-of-line photon event
// The environment of a photon event run out of line (the event form): the
// photon's stream, the product it pushes (every sampler pushes at most
// one) with the stream position at the push, its deposit (a photon event
// deposits at most once: below the cut-off), its step and crossing counts
// and error flags — all returned by value.
template <typename R>
struct PhotonEnv {
    static constexpr bool kInlineSamplers = true;
    Philox<R> rng;
    Part<R> q;
    uint32_t qpos;
    int nq;
    int dep_ir;
    R dep_e;
    int work, budget, ncross;
    unsigned flags;
    OMC_HD R uni() { return rng.uni(); }
    OMC_HD bool push(const Part<R> &x) {
        if (nq) {
            flags |= ERR_STACK;
            return false;
        }
        qpos = rng.position();
        q = x;
        nq = 1;
        return true;
    }
    OMC_HD void err(unsigned f) { flags |= f; }
    OMC_HD bool tick() { return ++work < budget; }
    OMC_HD void cross() { ncross++; }
    // one deposit record: a second deposit elsewhere would not fit it
    OMC_HD void deposit(int ir, R e) {
        if (dep_ir >= 0 && ir != dep_ir) flags |= ERR_LOG;
        dep_ir = ir;
        dep_e += e;
    }
};

template <typename R>
struct PhotonEventOut {
    Part<R> p;
    PhotonEnv<R> e;
    int alive;
};

// One photon event (delta tracking on uniform grids, else the voxel walk,
// then the interaction) compiled once, out of line, with its inputs and
// results by value: every kernel that runs photon events (the transport
// cycles and the drain) runs the same machine code for them, so they
// agree to the bit, and the calling kernel's particle and environment
// never have their address taken.
template <typename R>
OMC_COLD PhotonEventOut<R> photon_event_outline(const DevData<R> &D, Part<R> p, Philox<R> rng, int work,
                                                int budget) {
    PhotonEventOut<R> o;
    o.e.rng = rng;
    o.e.qpos = 0;
    o.e.nq = 0;
    o.e.dep_ir = -1;
    o.e.dep_e = R(0);
    o.e.work = work;
    o.e.budget = budget;
    o.e.ncross = 0;
    o.e.flags = 0;
    o.alive = (D.woodcock ? photon_step_delta(D, o.e, p) : photon_step(D, o.e, p)) ? 1 : 0;
    o.p = p;
    return o;
}

// Russian roulette of a photon made by an electron interaction when photons
// are split (ompmc.c:4169-4182, 4358-4371, 4647-4660): it survives with
// probability 1/nsplit and then carries nsplit times its weight; otherwise
// its weight and energy are zeroed (it deposits nothing).
template <typename R, typename Env>
OMC_HD void roulette(const DevData<R> &D, Env &g, Part<R> &q) {
    R rnno = g.uni();
    if (rnno * R(D.nsplit) > R(1)) {
        q.wt = R(0);
        q.e = R(0);
    } else {
        q.wt *= R(D.nsplit);
    }
}

// ---------------------------------------------- electron samplers (e+-)
// Annihilation at rest: two back-to-back photons of m each; p becomes the
// first and the second is pushed (rannih, ompmc.c:4129-4185).
template <typename R, typename Env>
OMC_HD void rannih(const DevData<R> &D, Env &g, Part<R> &p) {
    R rnno = g.uni();
    R costhe = R(2) * rnno - R(1);
    R sinthe = m_sqrt(m_max(R(0), (R(1) - costhe) * (R(1) + costhe)));
    (void)g.uni();
    R cphi, sphi;
    azimuth(g, cphi, sphi);
    p.e = R(D_RM);
    p.iq = 0;
    p.u = sinthe * cphi;
    p.v = sinthe * sphi;
    p.w = costhe;
    Part<R> q = p;
    q.u = -p.u;
    q.v = -p.v;
    q.w = -p.w;
    if (D.nsplit > 1) {
        roulette(D, g, p);
        roulette(D, g, q);
    }
    g.push(q);
}

// Bremsstrahlung: photon energy from the Bethe-Heitler screening rejection
// (Coulomb corrected above 50 MeV), photon angle from Koch-Motz 2BS
// (brems, ompmc.c:4188-4374).  p keeps its direction; the photon is pushed.
template <typename R, typename Env>
OMC_COLD void brems(const DevData<R> &D, Env &g, Part<R> &p) {
    const R RMr = R(D_RM);
    int imed = D.med[p.ir];
    const MedS<R> &M = D.ms[imed];
    R eie = p.e;
    int l = eie < R(50) ? 1 : 3, l1 = l + 1;
    R ekin = eie - RMr;
    R brmin = M.ap / ekin;
    R waux = -m_log(brmin);
    R a = p.u, b = p.v, c = p.w;
    R sinpsi = a * a + b * b, sindel = 0, cosdel = 0;
    if (sinpsi > R(1.0E-20)) {
        sinpsi = m_sqrt(sinpsi);
        sindel = b / sinpsi;
        cosdel = a / sinpsi;
    }
    R ztarg = M.zbrang;
    R tteie = eie / RMr;
    R beta = m_sqrt((tteie - R(1)) * (tteie + R(1))) / tteie;
    R y2max = R(2) * beta * (R(1) + beta) * tteie * tteie;
    R y2maxi = R(1) / y2max;
    R z2maxi = m_sqrt(y2max + R(1));
    R br, esg, ese, rejf, r7;
    int guard = 0;
    do {
        R r6 = g.uni();
        r7 = g.uni();
        br = brmin * m_exp(r6 * waux);
        esg = ekin * br;
        ese = eie - esg;
        R delta = esg / eie / ese * M.delcm;
        R aux = ese / eie;
        R phi1, phi2;
        if (delta < R(1)) {
            phi1 = M.dl1[l - 1] + delta * (M.dl2[l - 1] + delta * M.dl3[l - 1]);
            phi2 = M.dl1[l1 - 1] + delta * (M.dl2[l1 - 1] + delta * M.dl3[l1 - 1]);
        } else {
            phi1 = M.dl4[l - 1] + M.dl5[l - 1] * m_log(delta + M.dl6[l - 1]);
            phi2 = phi1;
        }
        rejf = (R(1) + aux * aux) * phi1 - R(2) * aux * phi2 / R(3);
        if (++guard > 100000) { g.err(ERR_LOOP); break; }
    } while (r7 >= rejf);
    Part<R> q = p;
    q.e = esg;
    q.iq = 0;
    R ttese = ese / RMr;
    R esedei = ttese / tteie;
    R rjarg1 = R(1) + esedei * esedei;
    R rjarg2 = rjarg1 + R(2) * esedei;
    R aux = R(2) * ese * tteie / esg;
    aux = aux * aux;
    R aux1 = aux * ztarg, rjarg3;
    if (aux1 > R(10)) rjarg3 = -m_log(M.zbrang) + (R(1) - aux1) / (aux1 * aux1);
    else rjarg3 = m_log(aux / (R(1) + aux1));
    R rejmax = rjarg1 * rjarg3 - rjarg2;
    R rtest = R(1), rejtst = R(0), y2tst = 0;
    guard = 0;
    while (rtest >= rejtst) {
        y2tst = g.uni();
        rtest = g.uni();
        R aux3 = z2maxi / (y2tst + (R(1) - y2tst) * z2maxi);
        rtest = rtest * aux3 * rejmax;
        y2tst = aux3 * aux3 - R(1);
        R a4 = sq(aux3 * aux3);
        R y2tst1 = esedei * y2tst / a4;
        R aux4 = R(16) * y2tst1 - rjarg2;
        R aux5 = rjarg1 - R(4) * y2tst1;
        if (rtest < aux4 + aux5 * rjarg3) break;
        R aux2 = m_log(aux / (R(1) + aux1 / a4));
        rejtst = aux4 + aux5 * aux2;
        if (++guard > 100000) { g.err(ERR_LOOP); break; }
    }
    R costhe = R(1) - R(2) * y2tst * y2maxi;
    R sinthe = m_sqrt(m_max(R(0), R(1) - costhe * costhe));
    R cphi, sphi;
    azimuth(g, cphi, sphi);
    if (sinpsi >= R(1.0E-10)) {
        R us = sinthe * cphi, vs = sinthe * sphi;
        q.u = c * cosdel * us - sindel * vs + a * costhe;
        q.v = c * sindel * us + cosdel * vs + b * costhe;
        q.w = c * costhe - sinpsi * us;
    } else {
        q.u = sinthe * cphi;
        q.v = sinthe * sphi;
        q.w = c * costhe;
    }
    p.e = ese;
    if (D.nsplit > 1) roulette(D, g, q);
    g.push(q);
}

// Moller scattering (moller, ompmc.c:4377-4453): p keeps energy ese1, the
// delta ray (ese2) is pushed.
template <typename R, typename Env>
OMC_COLD void moller(const DevData<R> &D, Env &g, Part<R> &p) {
    const R RMr = R(D_RM);
    const MedS<R> &M = D.ms[D.med[p.ir]];
    R eie = p.e, ekin = eie - RMr;
    if (ekin <= R(2) * M.te) return;
    R t0 = ekin / RMr, e0 = t0 + R(1);
    R extrae = eie - M.thmoll;
    R g2 = (t0 * t0) / (e0 * e0), g3 = (R(2) * t0 + R(1)) / (e0 * e0);
    R gmax = R(1) + R(1.25) * g2;
    R br, rejf4, r28;
    int guard = 0;
    do {
        R r27 = g.uni();
        br = M.te / (ekin - extrae * r27);
        R r = br / (R(1) - br);
        r28 = g.uni();
        rejf4 = R(1) + g2 * (br * br) + r * (r - g3);
        r28 *= gmax;
        if (++guard > 100000) { g.err(ERR_LOOP); break; }
    } while (r28 > rejf4);
    R ekse2 = br * ekin, ese1 = eie - ekse2, ese2 = ekse2 + RMr;
    p.e = ese1;
    R h1 = (eie + RMr) / ekin;
    R costh = h1 * (ese1 - RMr) / (ese1 + RMr);
    Uphi<R> h;
    uphi21(g, p, h, m_sqrt(costh), m_sqrt(R(1) - costh));
    costh = h1 * (ese2 - RMr) / (ese2 + RMr);
    Part<R> q = uphi32(p, h, m_sqrt(costh), -m_sqrt(R(1) - costh));
    q.e = ese2;
    q.iq = -1;
    g.push(q);
}

// Bhabha scattering (bhabha, ompmc.c:4456-4543): the more energetic
// particle stays the positron.
template <typename R, typename Env>
OMC_COLD void bhabha(const DevData<R> &D, Env &g, Part<R> &p) {
    const R RMr = R(D_RM);
    const MedS<R> &M = D.ms[D.med[p.ir]];
    R eip = p.e, ekin = eip - RMr;
    R t0 = ekin / RMr, e0 = t0 + R(1);
    R yy = R(1) / (t0 + R(2));
    R beta2 = (e0 * e0 - R(1)) / (e0 * e0);
    R ep0 = M.te / ekin, ep0c = R(1) - ep0;
    R yp = R(1) - R(2) * yy;
    R b4 = yp * yp * yp;
    R b3 = b4 + yp * yp;
    R b2 = yp * (R(3) + yy * yy);
    R b1 = R(2) - yy * yy;
    R br, r4, rejf2;
    int guard = 0;
    do {
        R r3 = g.uni();
        br = ep0 / (R(1) - ep0c * r3);
        r4 = g.uni();
        rejf2 = R(1) - beta2 * br * (b1 - br * (b2 - br * (b3 - br * b4)));
        if (++guard > 100000) { g.err(ERR_LOOP); break; }
    } while (r4 > rejf2);
    int iqnew;
    if (br < R(0.5)) {
        iqnew = -1;
    } else {
        p.iq = -1;
        iqnew = 1;
        br = R(1) - br;
    }
    br = m_max(br, R(0));
    R ekse2 = br * ekin, ese1 = eip - ekse2, ese2 = ekse2 + RMr;
    p.e = ese1;
    R h1 = (eip + RMr) / ekin;
    R costh = m_min(R(1), h1 * (ese1 - RMr) / (ese1 + RMr));
    Uphi<R> h;
    uphi21(g, p, h, m_sqrt(costh), m_sqrt(R(1) - costh));
    costh = h1 * (ese2 - RMr) / (ese2 + RMr);
    Part<R> q = uphi32(p, h, m_sqrt(costh), -m_sqrt(R(1) - costh));
    q.e = ese2;
    q.iq = iqnew;
    g.push(q);
}

// Two-photon annihilation in flight, Heitler (annih, ompmc.c:4546-4663).
template <typename R, typename Env>
OMC_COLD void annih(const DevData<R> &D, Env &g, Part<R> &p) {
    const R RMr = R(D_RM);
    R avip = p.e + RMr;
    R a = avip / RMr;
    R gg = a - R(1), t = gg - R(1), pp = m_sqrt(a * t);
    R pot = pp / t, ep0 = R(1) / (a + pp);
    R wsamp = m_log((R(1) - ep0) / ep0);
    R aa = p.u, bb = p.v, cc = p.w;
    R sinpsi = aa * aa + bb * bb, sindel = 0, cosdel = 0;
    if (sinpsi > R(1.0E-20)) {
        sinpsi = m_sqrt(sinpsi);
        sindel = bb / sinpsi;
        cosdel = aa / sinpsi;
    }
    R ep, r2, rejf;
    int guard = 0;
    do {
        R r1 = g.uni();
        ep = ep0 * m_exp(r1 * wsamp);
        r2 = g.uni();
        rejf = R(1) - sq(ep * a - R(1)) / (ep * (a * a - R(2)));
        if (++guard > 100000) { g.err(ERR_LOOP); break; }
    } while (r2 > rejf);
    R esg1 = avip * ep;
    p.e = esg1;
    p.iq = 0;
    R costhe = m_min(R(1), (esg1 - RMr) * pot / esg1);
    R sinthe = m_sqrt(R(1) - costhe * costhe);
    R cphi, sphi;
    azimuth(g, cphi, sphi);
    auto dir = [&](R ct, R st, R &u, R &v, R &w) {
        if (sinpsi >= R(1.0E-10)) {
            R us = st * cphi, vs = st * sphi;
            u = cc * cosdel * us - sindel * vs + aa * ct;
            v = cc * sindel * us + cosdel * vs + bb * ct;
            w = cc * ct - sinpsi * us;
        } else {
            u = st * cphi;
            v = st * sphi;
            w = cc * ct;
        }
    };
    dir(costhe, sinthe, p.u, p.v, p.w);
    Part<R> q = p;
    R esg2 = avip - esg1;
    q.e = esg2;
    costhe = m_min(R(1), (esg2 - RMr) * pot / esg2);
    sinthe = -m_sqrt(R(1) - costhe * costhe);
    dir(costhe, sinthe, q.u, q.v, q.w);
    if (D.nsplit > 1) {
        roulette(D, g, p);
        roulette(D, g, q);
    }
    g.push(q);
}

// ------------------------------------------- elastic scattering (e+-)
struct SpinIdx {
    int i, j;
};

// Mott/spin rejection function, linear in u = sqrt((1-cos)/2); the energy
// and q1 bins are drawn on first use and kept for the step
// (spinRejection, ompmc.c:3115-3185).  Indices are clamped to the table
// (the reference reads one element past a row at the edges).
template <typename R, typename Env>
OMC_HD R spin_rej(const DevData<R> &D, Env &g, int imed, int qel, R elke, R beta2, R q1, R cost, bool &spin_index,
                  bool is_single, SpinIdx &si) {
    if (spin_index) {
        spin_index = false;
        R ai;
        if (beta2 >= D.b2spin_min) {
            ai = (beta2 - D.b2spin_min) * D.dbeta2i;
            si.i = (int)ai;
            ai -= (R)si.i;
            si.i += 16;
        } else if (elke > D.espml) {
            ai = (elke - D.espml) * D.dleneri;
            si.i = (int)ai;
            ai -= (R)si.i;
        } else {
            si.i = 0;
            ai = R(-1);
        }
        R rnno = g.uni();
        if (rnno < ai) si.i += 1;
        if (is_single) {
            si.j = 0;
        } else {
            R qq1 = R(2) * q1;
            qq1 = qq1 / (R(1) + qq1);
            R aj = qq1 * D.dqq1i;
            si.j = (int)aj;
            if (si.j >= 15) {
                si.j = 15;
            } else {
                aj -= (R)si.j;
                rnno = g.uni();
                if (rnno < aj) si.j += 1;
            }
        }
    }
    R xi = m_sqrt(R(0.5) * (R(1) - cost));
    R ak = xi * R(31);
    int k = (int)ak;
    ak -= (R)k;
    if (k > 30) { k = 30; ak = R(1); }
    if (k < 0) { k = 0; ak = R(0); }
    int i = si.i < 0 ? 0 : (si.i > 31 ? 31 : si.i);
    int j = si.j < 0 ? 0 : (si.j > 15 ? 15 : si.j);
    const R *row = D.spin + ((((size_t)imed * 2 + qel) * D_NE1 + i) * D_NQ1 + j) * D_NU1;
    return (R(1) - ak) * row[k] + ak * row[k + 1];
}

struct MsIdx {
    int i, j;
};

// Multiple-scattering angle from the screened Rutherford x Mott
// distribution: no scattering, one or a few single scatterings (lambda <=
// 13.8), else the q^(2+) surface (mscat, ompmc.c:3624-3803).  quirk: the
// surface's in-bin slope du is ums[k]-ums[k] (zero), so u is one of the 32
// nodes; ref_compat = 0 uses ums[k+1]-ums[k].
template <typename R, typename Env>
OMC_HD void mscat(const DevData<R> &D, Env &g, int imed, int qel, bool &spin_index, bool &find_index, R elke, R beta2,
                  R q1, R lambda, R chia2, R &cost, R &sint, MsIdx &mi, R &omega2, SpinIdx &si) {
    R explambda = m_exp(-lambda);
    if (lambda <= R(13.8)) {
        R sprob = g.uni();
        if (sprob < explambda) {
            cost = R(1);
            sint = R(0);
            return;
        }
        R wsum = (R(1) + lambda) * explambda;
        if (sprob < wsum) {
            R xi, rejf, rnno;
            int guard = 0;
            do {
                xi = g.uni();
                xi = R(2) * chia2 * xi / (R(1) - xi + chia2);
                cost = R(1) - xi;
                rejf = spin_rej(D, g, imed, qel, elke, beta2, q1, cost, spin_index, false, si);
                rnno = g.uni();
                if (++guard > 100000) { g.err(ERR_LOOP); break; }
            } while (rnno > rejf);
            sint = m_sqrt(xi * (R(2) - xi));
            return;
        }
        if (lambda <= R(1)) {
            int icount = 0;
            R wprob = explambda;
            wsum = explambda;
            cost = R(1);
            sint = R(0);
            do {
                icount += 1;
                if (icount > 20) break;
                wprob = wprob * lambda / (R)icount;
                wsum = wsum + wprob;
                R xi, cosz, rejf, rnno;
                int guard = 0;
                do {
                    xi = g.uni();
                    xi = R(2) * chia2 * xi / (R(1) - xi + chia2);
                    cosz = R(1) - xi;
                    rejf = spin_rej(D, g, imed, qel, elke, beta2, q1, cosz, spin_index, false, si);
                    rnno = g.uni();
                    if (++guard > 100000) { g.err(ERR_LOOP); break; }
                } while (rnno > rejf);
                R sinz = xi * (R(2) - xi);
                if (sinz > R(1.0E-20)) {
                    sinz = m_sqrt(sinz);
                    xi = g.uni();
                    R phi = xi * R(6.2831853);
                    cost = cost * cosz - sint * sinz * m_cos(phi);
                    sint = m_sqrt(m_max(R(0), (R(1) - cost) * (R(1) + cost)));
                }
            } while (wsum <= sprob);
            return;
        }
    }
    if (lambda <= R(1.0E5)) {
        R llmbda = m_log(lambda);
        if (find_index) {
            R ai = llmbda * D.dllambi;
            mi.i = (int)ai;
            ai -= (R)mi.i;
            R xi = g.uni();
            if (xi < ai) mi.i += 1;
            if (q1 < R(1.0E-3)) {
                mi.j = 0;
            } else if (q1 < R(0.5)) {
                R aj = q1 * D.dqmsi;
                mi.j = (int)aj;
                aj -= (R)mi.j;
                xi = g.uni();
                if (xi < aj) mi.j += 1;
            } else {
                mi.j = 7;
            }
            if (llmbda < R(2.2299))
                omega2 = chia2 * (lambda + R(4)) *
                         (R(1.347006) + llmbda * (R(0.209364) - llmbda * (R(0.45525) - llmbda * (R(0.50142) - R(0.081234) * llmbda))));
            else
                omega2 = chia2 * (lambda + R(4)) *
                         (R(-2.77164) + llmbda * (R(2.94874) - llmbda * (R(0.1535754) - llmbda * R(0.00552888))));
            find_index = false;
        }
        int ii = mi.i < 0 ? 0 : (mi.i > 63 ? 63 : mi.i);
        int jj = mi.j < 0 ? 0 : (mi.j > 7 ? 7 : mi.j);
        const MsE<R> *row = D.msurf + (ii * 8 + jj) * 32;
        R xi, rejf, rnno;
        int guard = 0;
        do {
            xi = g.uni();
            R ak = xi * R(31);
            int k = (int)ak;
            ak -= (R)k;
            if (k > 30) k = 30;
            if (ak > row[k].w) k = row[k].i;
            if (k < 0) k = 0;
            if (k > 30) k = 30;
            R a = row[k].f, u = row[k].u;
            R du = D.ref_compat ? (row[k].u - u) : (row[k + 1].u - u);
            xi = g.uni();
            if (m_abs_lt(a, R(0.2))) {
                R x1 = R(0.5) * (R(1) - xi) * a;
                u += xi * du * (R(1) + x1 * (R(1) - xi * a));
            } else {
                u -= du / a * (R(1) - m_sqrt(R(1) + xi * a * (R(2) + a)));
            }
            xi = omega2 * u / (R(1) + R(0.5) * omega2 - u);
            if (xi > R(1.99999)) xi = R(1.99999);
            cost = R(1) - xi;
            rejf = spin_rej(D, g, imed, qel, elke, beta2, q1, cost, spin_index, false, si);
            rnno = g.uni();
            if (++guard > 100000) { g.err(ERR_LOOP); break; }
        } while (rnno > rejf);
        sint = m_sqrt(xi * (R(2) - xi));
    } else {
        // lambda beyond the surface: the reference leaves the angle unset;
        // no deflection here.
        cost = R(1);
        sint = R(0);
    }
}

// Single elastic scattering with spin rejection (sscat, ompmc.c:3188-3217).
template <typename R, typename Env>
OMC_HD void sscat(const DevData<R> &D, Env &g, int imed, int qel, R chia2, R elke, R beta2, R &cost, R &sint) {
    bool spin_index = true;
    SpinIdx si{0, 0};
    R xi, rejf, rnno;
    int guard = 0;
    do {
        xi = g.uni();
        xi = R(2) * chia2 * xi / (R(1) - xi + chia2);
        cost = R(1) - xi;
        rejf = spin_rej(D, g, imed, qel, elke, beta2, R(0), cost, spin_index, true, si);
        rnno = g.uni();
        if (++guard > 100000) { g.err(ERR_LOOP); break; }
    } while (rnno > rejf);
    sint = m_sqrt(xi * (R(2) - xi));
}

// PRESTA-II condensed-history step: two MS sub-steps, random hinge, energy
// loss corrections; returns the straight-line distance and the final
// position and direction (msdist, ompmc.c:3805-3994).
template <typename R, typename Env>
OMC_HD R msdist(const DevData<R> &D, Env &g, const Part<R> &p, int imed, int iq, R rhof, R de, R tustep, R eke,
                R &xf, R &yf, R &zf, R &uf, R &vf, R &wf) {
    const R RMr = R(D_RM);
    const MedS<R> &M = D.ms[imed];
    int qel = (1 + iq) / 2;
    R blccc = M.blcc, xcccc = M.xcc;
    R e = eke - R(0.5) * de;
    R tau = e / RMr, tau2 = tau * tau;
    R epsilon = de / eke, epsilonp = de / e;
    e *= (R(1) - (epsilonp * epsilonp) * (R(6) + R(10) * tau + R(5) * tau2) / (R(24) * tau2 + R(72) * tau + R(48)));
    R p2 = e * (e + R(2) * RMr);
    R beta2 = p2 / (p2 + RMr * RMr);
    R chia2 = xcccc / (R(4) * p2 * blccc);
    R lambda = R(0.5) * tustep * rhof * blccc / beta2;
    R tmp = epsilonp / ((tau + R(1)) * (tau + R(2)));
    R temp2 = R(0.166666) * (R(4) + tau * (R(6) + tau * (R(7) + tau * (R(4) + tau)))) * tmp * tmp;
    lambda *= (R(1) - temp2);
    R elke = m_log(e);
    int lelke = lidx(M.eke1, M.eke0, elke);
    if (lelke < 0) {
        lelke = 0;
        elke = (R(1) - M.eke0) / M.eke1;
    }
    const ElBin<R> &B = ebin(D, imed, qel, lelke);
    R etap = pwl(B.eta, elke);
    R xi_corr = pwl(B.q1c, elke);
    R gamma = pwl(B.q2c, elke);
    R ms_corr = pwl(B.blcce, elke);
    chia2 *= etap;
    lambda /= (etap * (R(1) + chia2));
    lambda *= ms_corr;
    R chilog = m_log(R(1) + R(1) / chia2);
    R q1 = R(2) * chia2 * (chilog * (R(1) + chia2) - R(1));
    gamma = R(6) * chia2 * (R(1) + chia2) * (chilog * (R(1) + R(2) * chia2) - R(2)) / q1 * gamma;
    R xi = q1 * lambda;
    bool find_index = true, spin_index = true;
    MsIdx mi{0, 0};
    SpinIdx si{0, 0};
    R omega2 = 0;
    R w1 = 0, sint1 = 0, w2 = 0, sint2 = 0, cphi1 = 0, sphi1 = 0, cphi2 = 0, sphi2 = 0;
    // the two sub-steps' deflections in that order, from one inlined copy
    // of mscat (the results are picked by name, not by a dynamic index,
    // so they stay in registers)
#pragma unroll 1
    for (int k = 0; k < 2; k++) {
        R w, st, cp, sp;
        mscat(D, g, imed, qel, spin_index, find_index, elke, beta2, xi, lambda, chia2, w, st, mi, omega2, si);
        azimuth(g, cp, sp);
        if (k == 0) {
            w1 = w; sint1 = st; cphi1 = cp; sphi1 = sp;
        } else {
            w2 = w; sint2 = st; cphi2 = cp; sphi2 = sp;
        }
    }
    R u2 = sint2 * cphi2, v2 = sint2 * sphi2;
    R u2p = w1 * u2 + sint1 * w2;
    R us = u2p * cphi1 - v2 * sphi1;
    R vs = u2p * sphi1 + v2 * cphi1;
    R ws = w1 * w2 - sint1 * u2;
    xi *= R(2) * xi_corr;
    R eta = g.uni();
    R eta1 = R(0.5) * (R(1) - eta);
    R delta = R(0.9082483) - (R(0.1020621) - R(0.0263747) * gamma) * xi;
    R temp1 = R(2) + tau;
    R temp = (R(2) + tau * temp1) / ((tau + R(1)) * temp1);
    temp -= (tau + R(1)) / ((tau + R(2)) * (chilog * (R(1) + chia2) - R(1)));
    temp *= epsilonp;
    temp1 = R(1) - temp;
    delta += R(0.40824829) * (epsilon * (tau + R(1)) /
                                  ((tau + R(2)) * (chilog * (R(1) + chia2) - R(1)) * (chilog * (R(1) + R(2) * chia2) - R(2))) -
                              R(0.25) * (temp * temp));
    R b = eta * delta, c = eta * (R(1) - delta);
    R w1v2 = w1 * v2;
    R ut = b * sint1 * cphi1 + c * (cphi1 * u2 - sphi1 * w1v2) + eta1 * us * temp1;
    R vt = b * sint1 * sphi1 + c * (sphi1 * u2 + cphi1 * w1v2) + eta1 * vs * temp1;
    R wt = eta1 * (R(1) + temp) + b * w1 + c * w2 + eta1 * ws * temp1;
    R ustep = tustep * m_sqrt(ut * ut + vt * vt + wt * wt);
    R u0 = p.u, v0 = p.v, w0 = p.w;
    R sint02 = u0 * u0 + v0 * v0;
    if (sint02 > R(1.0E-20)) {
        R sint0 = m_sqrt(sint02);
        R sint0i = R(1) / sint0;
        R cphi0 = sint0i * u0, sphi0 = sint0i * v0;
        u2p = w0 * us + sint0 * ws;
        ws = w0 * ws - sint0 * us;
        us = u2p * cphi0 - vs * sphi0;
        vs = u2p * sphi0 + vs * cphi0;
        u2p = w0 * ut + sint0 * wt;
        wt = w0 * wt - sint0 * ut;
        ut = u2p * cphi0 - vt * sphi0;
        vt = u2p * sphi0 + vt * cphi0;
    } else {
        wt = w0 * wt;
        ws = w0 * ws;
    }
    xf = p.x + tustep * ut;
    yf = p.y + tustep * vt;
    zf = p.z + tustep * wt;
    uf = us;
    vf = vs;
    wf = ws;
    return ustep;
}

// ------------------------------------------------------------ CSDA loss
// Path length from ekei down to ekef inside one interval of the log-linear
// stopping-power table (computeDrange, ompmc.c:3997-4033).
template <typename R>
OMC_OUTLINE R drange(const DevData<R> &D, int imed, int qel, int lelke, R ekei, R ekef, R elkei, R elkef) {
    R fedep = R(1) - ekef / ekei;
    R elktmp = R(0.5) * (elkei + elkef + R(0.25) * fedep * fedep * (R(1) + fedep * (R(1) + R(0.875) * fedep)));
    const ElBin<R> &B = ebin(D, imed, qel, lelke);
    R dedxmid = pwl(B.dedx, elktmp);
    dedxmid = R(1) / dedxmid;
    R aux = B.dedx.a1 * dedxmid;
    aux = aux * (R(1) + R(2) * aux) * fedep * fedep / (R(6) * (R(2) - fedep) * (R(2) - fedep));
    return fedep * ekei * dedxmid * (R(1) + aux);
}

// Energy lost to sub-threshold processes over path tustep (computeEloss,
// ompmc.c:4036-4126).
template <typename R>
OMC_OUTLINE R eloss(const DevData<R> &D, int imed, int qel, R rhof, R tustep, R range, R eke, R elke, int lelke) {
    const MedS<R> &M = D.ms[imed];
    R tuss = range - ebin(D, imed, qel, lelke).range / rhof;
    R de;
    if (tuss >= tustep) {
        const ElBin<R> &B = ebin(D, imed, qel, lelke);
        R dedxmid = pwl(B.dedx, elke);
        R aux = B.dedx.a1 / dedxmid;
        de = dedxmid * tustep * rhof;
        R fedep = de / eke;
        de *= (R(1) - R(0.5) * fedep * aux *
                          (R(1) - R(0.333333) * fedep * (aux - R(1) - R(0.25) * fedep * (R(2) - aux * (R(4) - aux)))));
    } else {
        int l = lelke;
        tuss = (range - tustep) * rhof;
        if (tuss <= R(0)) {
            de = eke - M.te * R(0.99);
        } else {
            while (l > 0 && tuss < ebin(D, imed, qel, l).range) l -= 1;
            R elktmp = ((R)(l + 2) - M.eke0) / M.eke1;
            const ElBin<R> &B1 = ebin(D, imed, qel, l + 1);
            R eketmp = B1.earr;
            tuss = (B1.range - tuss) / rhof;
            const ElBin<R> &B = ebin(D, imed, qel, l);
            R dedxmid = pwl(B.dedx, elktmp);
            R aux = B.dedx.a1 / dedxmid;
            de = dedxmid * tuss * rhof;
            R fedep = de / eketmp;
            de *= (R(1) - R(0.5) * fedep * aux *
                              (R(1) - R(0.333333) * fedep * (aux - R(1) - R(0.25) * fedep * (R(2) - aux * (R(4) - aux)))));
            de += eke - eketmp;
        }
    }
    return de;
}

// ------------------------------------------------------- electron step
enum EStep : int { E_DEAD = 0, E_ALIVE = 1, E_INTERACT = 2, E_END = 3 };

// The discrete interaction at the end of electron()'s transport loop
// (ompmc.c:5300-5451): bremsstrahlung or Moller (e-), bremsstrahlung,
// Bhabha or annihilation in flight (e+), by the branching ratios at the
// particle's energy (elke = ln of its kinetic energy, lelke its bin).
template <typename R, typename Env>
OMC_HD void electron_interact_at(const DevData<R> &D, Env &g, Part<R> &p, int imed, int qel, R elke, int lelke) {
    const ElBin<R> &B = ebin(D, imed, qel, lelke);
    if (p.iq < 0) {
        R ebr1 = pwl(B.br1, elke);
        R rnno = g.uni();
        if (rnno <= ebr1) {
            brems(D, g, p);
        } else if (p.e <= D.ms[imed].thmoll) {
            if (ebr1 <= R(0)) return;
            brems(D, g, p);
        } else {
            moller(D, g, p);
        }
    } else {
        R pbr1 = pwl(B.br1, elke);
        R rnno = g.uni();
        if (rnno < pbr1) {
            brems(D, g, p);
        } else {
            R pbr2 = pwl(B.br2, elke);
            if (rnno < pbr2) bhabha(D, g, p);
            else annih(D, g, p);
        }
    }
}

// The same for a particle left at its interaction site by electron_step
// (E_INTERACT): medium, energy and bin are recomputed from the particle
// exactly as the transport loop computed them.
template <typename R, typename Env>
OMC_HD void electron_interact(const DevData<R> &D, Env &g, Part<R> &p) {
    int imed = D.med[p.ir];
    const MedS<R> &M = D.ms[imed];
    R elke = m_log(p.e - R(D_RM));
    int lelke = lidx(M.eke1, M.eke0, elke);
    electron_interact_at(D, g, p, imed, (1 + p.iq) / 2, elke, lelke);
}

// Class II condensed-history transport of one electron() call with the
// fictitious cross-section method until the next discrete interaction, the
// cut-off or the phantom exit (electron, ompmc.c:4666-5451).  Returns
// E_END with the energy to deposit where the particle stands (cut-off: its
// kinetic energy, ompmc.c:4683-4705 and repeats; phantom exit: the
// reference's discard deposit), E_DEAD, E_ALIVE after the interaction, or
// with DEFER E_INTERACT when p stands at its discrete interaction.  Every
// cut-off site leaves p.e equal to the energy the reference tests (eie).
template <typename R, typename Env, bool DEFER>
OMC_HD int electron_transport(const DevData<R> &D, Env &g, Part<R> &p, R &edep_end) {
    const R RMr = R(D_RM);
    int irl = p.ir;
    int imed = D.med[irl];
    R rhof = D.rhof[irl];
    R eie = p.e;
    int iq = p.iq;
    int qel = (1 + iq) / 2;
    int medold = imed;
    if (eie <= ecut_of(D, irl)) {
        edep_end = p.e - RMr;
        return E_END;
    }

    R elke = 0;
    int lelke = 0;
    R sig0 = 0, demfp = 0, total_de = 0, total_tstep = 0;
    R ustep = 0;
    int guard = 0;
    for (;;) {  // tstep loop
        // The top of the tstep loop carries no state but the particle
        // (demfp is re-drawn here), so an event can stop after a budget of
        // iterations and resume in a later launch exactly where it was.
        if (!g.tstep_take()) return E_ALIVE;
        bool compute_tstep = true;
        R eke = eie - RMr;
        if (imed != -1) {
            const MedS<R> &M = D.ms[imed];
            R rnno = g.uni();
            if (rnno == R(0)) rnno = R(1.0E-30);
            demfp = m_max(-m_log(rnno), R(1.0E-5));
            elke = m_log(eke);
            lelke = lidx(M.eke1, M.eke0, elke);
            if (M.ismono[qel]) {
                const ElBin<R> &B = ebin(D, imed, qel, lelke);
                sig0 = pwl(B.sig, elke);
                R dedx0 = pwl(B.dedx, elke);
                sig0 /= dedx0;
            } else {
                sig0 = M.sige[qel];
            }
        }
        int nch = 0;            // condensed-history steps of this tstep iteration
        bool redraw = false;
        do {  // ustep loop
            if (D.chsteps > 0) {
                // after chsteps steps the remaining distance to the next
                // discrete interaction is drawn afresh at the top of the
                // tstep loop: the number of mean free paths to it is
                // exponential, hence memoryless, so the re-draw samples the
                // same distribution (the reference restarts after every
                // step, below; EGSnrc never)
                if (nch == D.chsteps) {
                    redraw = true;
                    break;
                }
                nch++;
            }
            if (++guard > 20000 || !g.tick()) { g.err(ERR_LOOP); return E_DEAD; }
            if (D.chsteps <= 0 && D.ref_compat) {
                // quirk: the reference declares total_tstep inside this loop
                // (ompmc.c:4799), so every step after the first of a tstep
                // cycle sees tstep = 0, takes a zero-length single-scattering
                // step (one draw) and restarts the cycle with a new demfp.
                total_tstep = R(0);
            }
            bool call_howfar, do_single = false, called_msdist = false;
            R tstep, tustep, de = 0, tvstep = 0, range = 0;
            R xf = 0, yf = 0, zf = 0, uf = 0, vf = 0, wf = 0;
            if (imed == -1) {
                tstep = R(1.0E9);
                ustep = tstep;
                tustep = ustep;
                call_howfar = true;
            } else {
                const MedS<R> &M = D.ms[imed];
                rhof = D.rhof[irl];
                if (sig0 <= R(0)) {
                    tstep = R(1.0E9);
                    sig0 = R(1.0E-15);
                } else {
                    if (compute_tstep) {
                        total_de = demfp / sig0;
                        R ekef = eke - total_de;
                        if (ekef <= ebin(D, imed, qel, 0).earr) {
                            tstep = R(1.0E9);
                        } else {
                            R elkef = m_log(ekef);
                            int lelkef = lidx(M.eke1, M.eke0, elkef);
                            if (lelkef == lelke) {
                                tstep = drange(D, imed, qel, lelke, eke, ekef, elke, elkef);
                            } else {
                                R ekei = ebin(D, imed, qel, lelke).earr;
                                R elkei = ((R)(lelke + 1) - M.eke0) / M.eke1;
                                R tuss = drange(D, imed, qel, lelke, eke, ekei, elke, elkei);
                                ekei = ebin(D, imed, qel, lelkef + 1).earr;
                                elkei = ((R)(lelkef + 2) - M.eke0) / M.eke1;
                                tstep = drange(D, imed, qel, lelkef, ekei, ekef, elkei, elkef);
                                tstep += tuss + ebin(D, imed, qel, lelke).range - ebin(D, imed, qel, lelkef + 1).range;
                            }
                        }
                        total_tstep = tstep;
                        compute_tstep = false;
                    }
                    tstep = total_tstep / rhof;
                }
                const ElBin<R> &B = ebin(D, imed, qel, lelke);
                R dedx0 = pwl(B.dedx, elke);
                R dedx = rhof * dedx0;
                R tmxs = pwl(B.tmxs, elke);
                tmxs /= rhof;
                R ekei = B.earr;
                R elkei = ((R)(lelke + 1) - M.eke0) / M.eke1;
                range = drange(D, imed, qel, lelke, eke, ekei, elke, elkei);
                range += B.range;
                range /= rhof;
                tustep = m_min(m_min(tstep, tmxs), range);
                R tperp = hownear(D, p);
                R blccl = rhof * M.blcc;
                R xccl = rhof * M.xcc;
                R p2 = eke * (eke + R(2) * RMr);
                R beta2 = p2 / (p2 + RMr * RMr);
                R etap = pwl(B.eta, elke);
                R ms_corr = pwl(B.blcce, elke);
                blccl = blccl / etap / (R(1) + R(0.25) * etap * xccl / blccl / p2) * ms_corr;
                R ssmfp = beta2 / blccl;
                R skindepth = R(3) * ssmfp;
                tustep = m_min(tustep, m_max(tperp, skindepth));
                if ((tustep <= tperp) && (tustep > skindepth)) {
                    call_howfar = false;
                    do_single = false;
                    called_msdist = true;
                    de = eloss(D, imed, qel, rhof, tustep, range, eke, elke, lelke);
                    tvstep = tustep;
                    ustep = msdist(D, g, p, imed, iq, rhof, de, tustep, eke, xf, yf, zf, uf, vf, wf);
                } else {
                    called_msdist = false;
                    R rnno = g.uni();
                    if (rnno < R(1.0E-30)) rnno = R(1.0E-30);
                    R lambda = -m_log(R(1) - rnno);
                    R lambda_max = R(0.5) * blccl * RMr / dedx;
                    R gg = eke / RMr + R(1);
                    lambda_max *= gg * gg * gg;
                    if (lambda >= R(0) && lambda_max > R(0)) {
                        R tuss;
                        if (lambda < lambda_max) tuss = lambda * ssmfp * (R(1) - R(0.5) * lambda / lambda_max);
                        else tuss = R(0.5) * lambda * ssmfp;
                        if (tuss < tustep) {
                            tustep = tuss;
                            do_single = true;
                        } else {
                            do_single = false;
                        }
                    } else {
                        // quirk: the particle is dropped without a deposit
                        g.err(ERR_LAMBDA);
                        return E_DEAD;
                    }
                    ustep = tustep;
                    call_howfar = !(ustep < tperp);
                }
            }
            int irold = p.ir, irnew = p.ir, idisc = 0;
            if (call_howfar) howfar(D, p, idisc, irnew, ustep);
            if (idisc > 0) {
                edep_end = iq > 0 ? p.e + RMr : p.e - RMr;
                return E_END;
            }
            if (ustep < R(0)) ustep = R(0);
            if (ustep == R(0) || imed == -1) {
                if (ustep != R(0)) {
                    R vstep = ustep;
                    p.x += p.u * vstep;
                    p.y += p.v * vstep;
                    p.z += p.w * vstep;
                }
                if (irnew != irold) {
                    p.ir = irnew;
                    irl = irnew;
                    imed = D.med[irl];
                    g.cross();
                }
                if (eie <= ecut_of(D, irl)) {
                    edep_end = p.e - RMr;
                    return E_END;
                }
                break;
            }
            R vstep = ustep;
            if (call_howfar) {
                tvstep = vstep;
                if (tvstep != tustep) do_single = false;
                de = eloss(D, imed, qel, rhof, tvstep, range, eke, elke, lelke);
            } else {
                tvstep = tustep;
                if (!called_msdist) de = eloss(D, imed, qel, rhof, tvstep, range, eke, elke, lelke);
            }
            R edep = de;
            R ekef = eke - de;
            R sinthe = 0, costhe = 1;
            if (!called_msdist) {
                if (do_single) {
                    const MedS<R> &M = D.ms[imed];
                    R ekems = m_max(ekef, ecut_of(D, irl) - RMr);
                    R p2 = ekems * (ekems + R(2) * RMr);
                    R beta2 = p2 / (p2 + RMr * RMr);
                    R chia2 = M.xcc / (R(4) * M.blcc * p2);
                    R elkems = m_log(ekems);
                    int lelkems = lidx(M.eke1, M.eke0, elkems);
                    R etap = pwl(ebin(D, imed, qel, lelkems).eta, elkems);
                    chia2 *= etap;
                    sscat(D, g, imed, qel, chia2, elkems, beta2, costhe, sinthe);
                } else {
                    sinthe = R(0);
                    costhe = R(1);
                }
                xf = p.x + p.u * vstep;
                yf = p.y + p.v * vstep;
                zf = p.z + p.w * vstep;
                if (do_single) {
                    Uphi<R> h;
                    uphi21(g, p, h, costhe, sinthe);
                }
                uf = p.u;
                vf = p.v;
                wf = p.w;
            }
            g.deposit(p.ir, p.wt * edep);
            p.x = xf; p.y = yf; p.z = zf;
            p.u = uf; p.v = vf; p.w = wf;
            renorm_dir(p.u, p.v, p.w);
            irold = p.ir;
            eie -= edep;
            p.e = eie;
            if (irnew == irl && eie <= ecut_of(D, irl)) {
                edep_end = p.e - RMr;
                return E_END;
            }
            medold = imed;
            if (imed != -1) {
                const MedS<R> &M = D.ms[imed];
                eke = eie - RMr;
                elke = m_log(eke);
                lelke = lidx(M.eke1, M.eke0, elke);
            }
            if (irnew != irold) {
                p.ir = irnew;
                irl = irnew;
                imed = D.med[irl];
                g.cross();
            }
            if (eie <= ecut_of(D, irl)) {
                edep_end = p.e - RMr;
                return E_END;
            }
            if (imed != medold) break;
            demfp -= de * sig0;
            total_de -= de;
            total_tstep -= tvstep * rhof;
            if (total_tstep < R(1.0E-9)) demfp = R(0);
        } while (demfp >= R(1.0E-5));
        if (redraw || (imed != medold) || (ustep == R(0)) || (imed == -1)) continue;
        const ElBin<R> &B = ebin(D, imed, qel, lelke);
        R sigf = pwl(B.sig, elke);
        R dedx0 = pwl(B.dedx, elke);
        sigf /= dedx0;
        R sigratio = sigf / sig0;
        R rfict = g.uni();
        if (!(rfict >= sigratio)) break;
    }
    // discrete interaction: here, or (DEFER) in a later kernel that runs
    // electron_interact on the particle as it stands
    if (DEFER) return E_INTERACT;
    electron_interact_at(D, g, p, imed, qel, elke, lelke);
    return E_ALIVE;
}

// One call of electron(): the transport above, then the local deposit where
// it ends (a positron annihilates at rest there when the deposit is below
// its energy, ompmc.c:4683-4705).  One deposit site and no call that takes
// the particle's or the environment's address: both stay in registers in
// the transport kernels.  Returns E_ALIVE when p (possibly changed into
// another particle) stays on the stack; with DEFER, E_INTERACT when p
// stands at its discrete interaction (electron_interact samples it).
template <typename R, typename Env, bool DEFER = false>
OMC_HD int electron_step(const DevData<R> &D, Env &g, Part<R> &p) {
    R edep = 0;
    const int r = electron_transport<R, Env, DEFER>(D, g, p, edep);
    if (r != E_END) return r;
    g.deposit(p.ir, p.wt * edep);
    if (p.iq > 0 && edep < p.e) {
        rannih(D, g, p);
        return E_ALIVE;
    }
    return E_DEAD;
}

}  // namespace omc
