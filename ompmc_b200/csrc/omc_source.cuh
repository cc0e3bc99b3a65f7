// Primary particles of the two ucodes.
#pragma once
#include "omc_physics.cuh"

namespace omc {

// Energy from the spectrum inverse CDF, or the mono-energetic value
// (omc_dosxyz.c:979-993).
template <typename R, typename G>
OMC_HD R source_energy(G &g, int spectrum, R energy, const R *cdf1, const R *cdf2, R deltak) {
    if (!spectrum) return energy;
    R r1 = g.uni(), r2 = g.uni();
    R kk = deltak * r1;
    if (kk > deltak - R(1)) kk = deltak - R(1);
    int k = (int)kk;
    return cdf1[k] + r2 * cdf2[k];
}

// Collimated point source at SSD on the z axis, cos^3 rejection over the
// collimator rectangle, starting on the z = zmin face
// (initHistory, omc_dosxyz.c:964-1068).
template <typename R, typename G>
OMC_HD Part<R> beam_primary(const DevData<R> &D, const BeamSrc<R> &S, G &g, R &ein) {
    Part<R> p;
    p.iq = S.charge;
    ein = source_energy(g, S.spectrum, S.energy, S.cdf1, S.cdf2, S.deltak);
    p.e = S.charge != 0 ? ein + R(D_RM) : ein;
    R rxyz;
    if (S.xsize == R(0) || S.ysize == R(0)) {
        p.x = S.xinl;
        p.y = S.yinl;
        rxyz = m_sqrt(S.ssd * S.ssd + p.x * p.x + p.y * p.y);
        p.w = S.ssd / rxyz;
    } else {
        R r3, fw;
        int guard = 0;
        do {
            r3 = g.uni();
            p.x = r3 * S.xsize + S.xinl;
            r3 = g.uni();
            p.y = r3 * S.ysize + S.yinl;
            r3 = g.uni();
            rxyz = m_sqrt(S.ssd * S.ssd + p.x * p.x + p.y * p.y);
            p.w = S.ssd / rxyz;
            fw = p.w * p.w * p.w;
        } while (r3 >= fw && ++guard < 100000);
    }
    p.z = D.zb[0];
    p.u = p.x / rxyz;
    p.v = p.y / rxyz;
    int ix, iy;
    if (S.xsize == R(0)) {
        ix = S.ixinl;
    } else {
        ix = S.ixinl - 1;
        while (D.xb[ix + 1] < p.x && ix < D.nx - 1) ix++;
    }
    if (S.ysize == R(0)) {
        iy = S.iyinl;
    } else {
        iy = S.iyinl - 1;
        while (D.yb[iy + 1] < p.y && iy < D.ny - 1) iy++;
    }
    if (ix < 0) ix = 0;
    if (iy < 0) iy = 0;
    p.ir = 1 + ix + iy * D.nx;
    p.wt = R(1);
    return p;
}

// matRad beamlet: uniform point on the bixel parallelogram, direction from
// the beam source (point, or a Gaussian spot in the bixel plane by
// Box-Muller), moved back along the ray to the phantom's bounding box and
// clamped inside (initHistory(ibeamlet), omc_matrad.c:1177-1413).
// quirk (ref_compat): the z clamp below zmin uses ybounds[0].
template <typename R, typename G>
OMC_HD Part<R> beamlet_primary(const DevData<R> &D, const BeamletSrc<R> &S, int ib, G &g, R &ein) {
    Part<R> p;
    p.iq = S.charge;
    ein = source_energy(g, S.spectrum, S.energy, S.cdf1, S.cdf2, S.deltak);
    p.e = S.charge != 0 ? ein + R(D_RM) : ein;
    R r1 = g.uni(), r2 = g.uni();
    const R *c = S.corner + 3 * ib, *s1 = S.side1 + 3 * ib, *s2 = S.side2 + 3 * ib;
    R xiso = r1 * s1[0] + r2 * s2[0] + c[0];
    R yiso = r1 * s1[1] + r2 * s2[1] + c[1];
    R ziso = r1 * s1[2] + r2 * s2[2] + c[2];
    int ibeam = S.ibeam[ib];
    R sx = S.src[3 * ibeam], sy = S.src[3 * ibeam + 1], sz = S.src[3 * ibeam + 2];
    if (S.gaussian) {
        R n1 = m_sqrt(s1[0] * s1[0] + s1[1] * s1[1] + s1[2] * s1[2]);
        R n2 = m_sqrt(s2[0] * s2[0] + s2[1] * s2[1] + s2[2] * s2[2]);
        R a = g.uni(), b = g.uni();
        R rr = m_sqrt(R(-2) * m_log(a));
        R th = R(2) * R(M_PI) * b;
        R g0 = rr * m_cos(th) * S.gauss_width, g1 = rr * m_sin(th) * S.gauss_width;
        sx += g0 * s1[0] / n1 + g1 * s2[0] / n2;
        sy += g0 * s1[1] / n1 + g1 * s2[1] / n2;
        sz += g0 * s1[2] / n1 + g1 * s2[2] / n2;
    }
    R xd = xiso - sx, yd = yiso - sy, zd = ziso - sz;
    R vn = m_sqrt(xd * xd + yd * yd + zd * zd);
    R u = -(xd) / vn, v = -(yd) / vn, w = -(zd) / vn;
    R ustep = R(sizeof(R) == 8 ? 1.7976931348623157e308 : 3.4028234663852886e38);
    R dist;
    if (u > R(0)) { dist = (D.xb[D.nx] - xiso) / u; if (dist < ustep) ustep = dist; }
    if (u < R(0)) { dist = -(xiso - D.xb[0]) / u; if (dist < ustep) ustep = dist; }
    if (v > R(0)) { dist = (D.yb[D.ny] - yiso) / v; if (dist < ustep) ustep = dist; }
    if (v < R(0)) { dist = -(yiso - D.yb[0]) / v; if (dist < ustep) ustep = dist; }
    if (w > R(0)) { dist = (D.zb[D.nz] - ziso) / w; if (dist < ustep) ustep = dist; }
    if (w < R(0)) { dist = -(ziso - D.zb[0]) / w; if (dist < ustep) ustep = dist; }
    p.x = xiso + ustep * u;
    p.y = yiso + ustep * v;
    p.z = ziso + ustep * w;
    p.u = -u;
    p.v = -v;
    p.w = -w;
    const R tiny = R(2) * R(sizeof(R) == 8 ? 2.2250738585072014e-308 : 1.1754943508222875e-38);
    if (p.x < D.xb[0]) p.x = D.xb[0] + tiny;
    if (p.x > D.xb[D.nx]) p.x = D.xb[D.nx] - tiny;
    if (p.y < D.yb[0]) p.y = D.yb[0] + tiny;
    if (p.y > D.yb[D.ny]) p.y = D.yb[D.ny] - tiny;
    if (p.z < D.zb[0]) p.z = (D.ref_compat ? D.yb[0] : D.zb[0]) + tiny;
    if (p.z > D.zb[D.nz]) p.z = D.zb[D.nz] - tiny;
    int ix = 0, iy = 0, iz = 0;
    while (ix < D.nx - 1 && D.xb[ix + 1] < p.x) ix++;
    while (iy < D.ny - 1 && D.yb[iy + 1] < p.y) iy++;
    while (iz < D.nz - 1 && D.zb[iz + 1] < p.z) iz++;
    p.ir = 1 + ix + iy * D.nx + iz * D.nx * D.ny;
    p.wt = R(1);
    return p;
}

}  // namespace omc
