/*
 * Oracle harness around the UNMODIFIED ompMC reference (test infrastructure
 * only; never linked into the product).
 *
 * The Makefile in this directory compiles, from the reference tree,
 *   src/ompmc.c, src/omc_utilities.c            as they are,
 *   src/omc_random.c     with -DsetRandom=ranmar_setRandom,
 *   ucodes/omc_dosxyz/omc_dosxyz.c with -Dmain=omc_dosxyz_ref_main
 *                                       -Dausgab=ref_ausgab,
 * and links this file, which supplies the two renamed link-time hooks:
 *   - setRandom() (omc_random.h:69-77): RANMAR by default; can record the
 *     stream each history consumes, or replay a scripted stream;
 *   - ausgab() (ompmc.h:39, omc_dosxyz.c:683-694): logs every deposit
 *     (region, weighted energy) and forwards to the reference tally.
 * The harness runs single-threaded (built without OpenMP), so a history is
 * exactly the sequence shower() executes on one stack.
 *
 * Exported entry points (called from Python through ctypes):
 *   h_init(inp_base)            parse `<inp_base>.inp` and run every init the
 *                               CLI runs before its batch loop
 *                               (omc_dosxyz.c:1150-1192)
 *   h_table(name, &n)           pointer + length of a reference table
 *   h_howfar / h_hownear        the reference geometry on a given state
 *   h_run(...)                  run histories; record random streams and
 *                               deposit sequences per history
 *   h_replay(...)               run one history on a scripted stream
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ompmc.h"
#include "omc_random.h"
#include "omc_utilities.h"

int verbose_flag = 0;   /* declared by omc_utilities.h:64, never defined by omc_dosxyz */

/* Symbols of omc_dosxyz.c (compiled as a library) */
struct Geom {
    int *med_indices;
    double *med_densities;
    int isize, jsize, ksize;
    double *xbounds, *ybounds, *zbounds;
};
extern struct Geom geometry;
void initPhantom(void);
void initSource(void);
void initScore(void);
void initHistory(void);
void ref_ausgab(double edep);
double ranmar_setRandom(void);

/* ---------------------------------------------------------------- RNG hook */
static int rng_mode = 0;          /* 0 RANMAR, 1 RANMAR + record, 2 replay */
static double *rn_buf = NULL;     /* record target or replay source */
static long rn_cap = 0, rn_pos = 0;
static int rn_overflow = 0;

/* Optional draw log: the function that called setRandom for each draw. */
static const char **draw_site = NULL;
static long draw_cap = 0;

double setRandom(void) {
    if (draw_site && rn_pos < draw_cap) {
        Dl_info info;
        void *ra = __builtin_return_address(0);
        draw_site[rn_pos] = (dladdr(ra, &info) && info.dli_sname) ? info.dli_sname : "?";
    }
    if (rng_mode == 2) {
        if (rn_pos < rn_cap) return rn_buf[rn_pos++];
        rn_overflow = 1;
        return 0.5;
    }
    double r = ranmar_setRandom();
    if (rng_mode == 1) {
        if (rn_pos < rn_cap) rn_buf[rn_pos] = r; else rn_overflow = 1;
        rn_pos++;
    }
    return r;
}

/* ------------------------------------------------------------- ausgab hook */
static int dep_log_on = 0;
static int *dep_ir = NULL;
static double *dep_e = NULL;
static long dep_cap = 0, dep_pos = 0;
static int dep_overflow = 0;
static long *dep_rnpos = NULL;   /* optional: random numbers drawn before each deposit */

void ausgab(double edep) {
    if (dep_log_on) {
        if (dep_pos < dep_cap) {
            dep_ir[dep_pos] = stack.ir[stack.np];
            dep_e[dep_pos] = stack.wt[stack.np] * edep;
            if (dep_rnpos) dep_rnpos[dep_pos] = rn_pos;
        } else {
            dep_overflow = 1;
        }
        dep_pos++;
    }
    ref_ausgab(edep);
}

/* ------------------------------------------------------------------ init */
int h_init(const char *inp_base) {
    static char name[512];
    strncpy(name, inp_base, sizeof(name) - 1);
    input_idx = 0;
    parseInputFile(name);
    initPhantom();
    initMediaData();
    initSource();
    initRegions();
    initVrt();
    initScore();
    initRandom();
    initStack();
    return 0;
}

int h_nvox(void) { return geometry.isize * geometry.jsize * geometry.ksize; }
int h_nmed(void) { return media.nmed; }

/* Reference tables by name, as flat arrays.  `n` receives the element count. */
/* Leading members of omc_dosxyz.c's struct Source (omc_dosxyz.c:342-352),
   declared here in the same order so the harness can read the inverse CDF
   of the spectrum the reference built in initSource (omc_dosxyz.c:478-502). */
struct SourceHead {
    int spectrum;
    int charge;
    double energy;
    double deltak;
    double *cdfinv1;
    double *cdfinv2;
};
extern struct SourceHead source;

const void *h_table(const char *t, long *n) {
    int nmed = media.nmed;
#define T(NAME, PTR, COUNT) if (strcmp(t, NAME) == 0) { *n = (COUNT); return (const void *)(PTR); }
    T("ge0", photon_data.ge0, nmed) T("ge1", photon_data.ge1, nmed)
    T("gmfp0", photon_data.gmfp0, nmed * MXGE) T("gmfp1", photon_data.gmfp1, nmed * MXGE)
    T("gbr10", photon_data.gbr10, nmed * MXGE) T("gbr11", photon_data.gbr11, nmed * MXGE)
    T("gbr20", photon_data.gbr20, nmed * MXGE) T("gbr21", photon_data.gbr21, nmed * MXGE)
    T("cohe0", photon_data.cohe0, nmed * MXGE) T("cohe1", photon_data.cohe1, nmed * MXGE)
    T("xgrid", rayleigh_data.xgrid, nmed * MXRAYFF) T("fcum", rayleigh_data.fcum, nmed * MXRAYFF)
    T("b_array", rayleigh_data.b_array, nmed * MXRAYFF) T("c_array", rayleigh_data.c_array, nmed * MXRAYFF)
    T("pmax0", rayleigh_data.pmax0, nmed * MXGE) T("pmax1", rayleigh_data.pmax1, nmed * MXGE)
    T("i_array", rayleigh_data.i_array, nmed * RAYCDFSIZE)
    T("dl1", pair_data.dl1, nmed * 8) T("dl2", pair_data.dl2, nmed * 8) T("dl3", pair_data.dl3, nmed * 8)
    T("dl4", pair_data.dl4, nmed * 8) T("dl5", pair_data.dl5, nmed * 8) T("dl6", pair_data.dl6, nmed * 8)
    T("bpar0", pair_data.bpar0, nmed) T("bpar1", pair_data.bpar1, nmed)
    T("delcm", pair_data.delcm, nmed) T("zbrang", pair_data.zbrang, nmed)
    T("esig0", electron_data.esig0, nmed * MXEKE) T("esig1", electron_data.esig1, nmed * MXEKE)
    T("psig0", electron_data.psig0, nmed * MXEKE) T("psig1", electron_data.psig1, nmed * MXEKE)
    T("ededx0", electron_data.ededx0, nmed * MXEKE) T("ededx1", electron_data.ededx1, nmed * MXEKE)
    T("pdedx0", electron_data.pdedx0, nmed * MXEKE) T("pdedx1", electron_data.pdedx1, nmed * MXEKE)
    T("ebr10", electron_data.ebr10, nmed * MXEKE) T("ebr11", electron_data.ebr11, nmed * MXEKE)
    T("pbr10", electron_data.pbr10, nmed * MXEKE) T("pbr11", electron_data.pbr11, nmed * MXEKE)
    T("pbr20", electron_data.pbr20, nmed * MXEKE) T("pbr21", electron_data.pbr21, nmed * MXEKE)
    T("tmxs0", electron_data.tmxs0, nmed * MXEKE) T("tmxs1", electron_data.tmxs1, nmed * MXEKE)
    T("blcce0", electron_data.blcce0, nmed * MXEKE) T("blcce1", electron_data.blcce1, nmed * MXEKE)
    T("etae_ms0", electron_data.etae_ms0, nmed * MXEKE) T("etae_ms1", electron_data.etae_ms1, nmed * MXEKE)
    T("etap_ms0", electron_data.etap_ms0, nmed * MXEKE) T("etap_ms1", electron_data.etap_ms1, nmed * MXEKE)
    T("q1ce_ms0", electron_data.q1ce_ms0, nmed * MXEKE) T("q1ce_ms1", electron_data.q1ce_ms1, nmed * MXEKE)
    T("q1cp_ms0", electron_data.q1cp_ms0, nmed * MXEKE) T("q1cp_ms1", electron_data.q1cp_ms1, nmed * MXEKE)
    T("q2ce_ms0", electron_data.q2ce_ms0, nmed * MXEKE) T("q2ce_ms1", electron_data.q2ce_ms1, nmed * MXEKE)
    T("q2cp_ms0", electron_data.q2cp_ms0, nmed * MXEKE) T("q2cp_ms1", electron_data.q2cp_ms1, nmed * MXEKE)
    T("range_ep", electron_data.range_ep, 2 * nmed * MXEKE)
    T("e_array", electron_data.e_array, nmed * MXEKE)
    T("eke0", electron_data.eke0, nmed) T("eke1", electron_data.eke1, nmed)
    T("sig_ismonotone", electron_data.sig_ismonotone, 2 * nmed)
    T("esig_e", electron_data.esig_e, nmed) T("psig_e", electron_data.psig_e, nmed)
    T("xcc", electron_data.xcc, nmed) T("blcc", electron_data.blcc, nmed)
    T("expeke1", electron_data.expeke1, nmed)
    T("spin_rej", spin_data.spin_rej, nmed * 2 * (MXE_SPIN1 + 1) * (MXQ_SPIN + 1) * (MXU_SPIN + 1))
    T("ums", mscat_data.ums_array, (MXL_MS + 1) * (MXQ_MS + 1) * (MXU_MS + 1))
    T("fms", mscat_data.fms_array, (MXL_MS + 1) * (MXQ_MS + 1) * (MXU_MS + 1))
    T("wms", mscat_data.wms_array, (MXL_MS + 1) * (MXQ_MS + 1) * (MXU_MS + 1))
    T("ims", mscat_data.ims_array, (MXL_MS + 1) * (MXQ_MS + 1) * (MXU_MS + 1))
    T("rho", pegs_data.rho, nmed) T("rlc", pegs_data.rlc, nmed)
    T("ae", pegs_data.ae, nmed) T("ap", pegs_data.ap, nmed)
    T("ue", pegs_data.ue, nmed) T("up", pegs_data.up, nmed)
    T("te", pegs_data.te, nmed) T("thmoll", pegs_data.thmoll, nmed)
    T("meke", pegs_data.meke, nmed)
    T("region_med", region.med, h_nvox() + 1) T("region_rhof", region.rhof, h_nvox() + 1)
    T("region_pcut", region.pcut, h_nvox() + 1) T("region_ecut", region.ecut, h_nvox() + 1)
    T("cdfinv1", source.cdfinv1, source.spectrum ? (long)source.deltak : 0)
    T("cdfinv2", source.cdfinv2, source.spectrum ? (long)source.deltak : 0)
#undef T
    *n = 0;
    return NULL;
}

/* Scalars of the spin and MS tables */
void h_spin_scalars(double *out) {
    out[0] = spin_data.b2spin_min; out[1] = spin_data.dbeta2i; out[2] = spin_data.espml;
    out[3] = spin_data.dleneri; out[4] = spin_data.dqq1i;
    out[5] = mscat_data.dllambi; out[6] = mscat_data.dqmsi;
}

/* ------------------------------------------------------------- geometry */
static void set_top(double x, double y, double z, double u, double v, double w, int ir) {
    stack.np = 0;
    stack.x[0] = x; stack.y[0] = y; stack.z[0] = z;
    stack.u[0] = u; stack.v[0] = v; stack.w[0] = w;
    stack.ir[0] = ir; stack.wt[0] = 1.0; stack.iq[0] = 0; stack.dnear[0] = 0.0;
}

/* One call of the reference howfar on the given state. */
void h_howfar(double x, double y, double z, double u, double v, double w, int ir,
              double ustep_in, double *ustep_out, int *irnew, int *idisc) {
    set_top(x, y, z, u, v, w, ir);
    int id = 0, irn = ir;
    double us = ustep_in;
    howfar(&id, &irn, &us);
    *ustep_out = us; *irnew = irn; *idisc = id;
}

double h_hownear(double x, double y, double z, int ir) {
    set_top(x, y, z, 0.0, 0.0, 1.0, ir);
    return hownear();
}

/* Straight-line walk until the particle leaves the phantom, mirroring the
   photon transport loop with an infinite interaction distance
   (ompmc.c:1969-2037): ustep = 1e8 -> howfar -> move -> region change.
   Records ustep, irnew and idisc of every call; returns the number of
   calls (capped at cap). */
int h_walk(double x, double y, double z, double u, double v, double w, int ir,
           int cap, double *ustep, int *irnew, int *idisc) {
    set_top(x, y, z, u, v, w, ir);
    int n = 0;
    while (n < cap) {
        int id = 0, irn = stack.ir[0];
        double us = 1.0E8;
        howfar(&id, &irn, &us);
        ustep[n] = us; irnew[n] = irn; idisc[n] = id;
        n++;
        if (id > 0) break;
        stack.x[0] += us * stack.u[0];
        stack.y[0] += us * stack.v[0];
        stack.z[0] += us * stack.w[0];
        stack.ir[0] = irn;
    }
    return n;
}

/* ------------------------------------------------------------- histories */
/* Source particle of the next history (initHistory, omc_dosxyz.c:964-1068)
   with RANMAR; fills q[11] = x,y,z,u,v,w,e,wt,ir,iq,dnear. */
void h_source(double *q) {
    initHistory();
    q[0] = stack.x[0]; q[1] = stack.y[0]; q[2] = stack.z[0];
    q[3] = stack.u[0]; q[4] = stack.v[0]; q[5] = stack.w[0];
    q[6] = stack.e[0]; q[7] = stack.wt[0]; q[8] = stack.ir[0]; q[9] = stack.iq[0];
    q[10] = stack.dnear[0];
}

/* Run `nhist` histories of the configured source with RANMAR.  For each
   history h records its primary (prim[11*h..]), the random numbers it
   consumed (rn[rn_off[h] .. rn_off[h+1]) and its deposits
   (dep_ir/dep_e[d_off[h] .. d_off[h+1])).  Returns 0, or -1 when a buffer
   overflowed. */
int h_run(int nhist, double *prim, double *rn, long rn_capacity, long *rn_off,
          int *dir, double *de, long d_capacity, long *d_off) {
    rn_buf = rn; rn_cap = rn_capacity; rn_pos = 0; rn_overflow = 0;
    dep_ir = dir; dep_e = de; dep_cap = d_capacity; dep_pos = 0; dep_overflow = 0;
    for (int h = 0; h < nhist; h++) {
        rn_off[h] = rn_pos;
        d_off[h] = dep_pos;
        rng_mode = 0;
        dep_log_on = 0;
        initHistory();
        double *q = prim + 11 * h;
        q[0] = stack.x[0]; q[1] = stack.y[0]; q[2] = stack.z[0];
        q[3] = stack.u[0]; q[4] = stack.v[0]; q[5] = stack.w[0];
        q[6] = stack.e[0]; q[7] = stack.wt[0]; q[8] = stack.ir[0]; q[9] = stack.iq[0];
        q[10] = stack.dnear[0];
        rng_mode = 1;
        dep_log_on = 1;
        shower();
    }
    rn_off[nhist] = rn_pos;
    d_off[nhist] = dep_pos;
    rng_mode = 0;
    dep_log_on = 0;
    return (rn_overflow || dep_overflow) ? -1 : 0;
}

/* Run one history from primary q[11] on the scripted stream rn[0..n).
   Records deposits; returns the count of random numbers consumed, or -1 on
   buffer overflow (stream exhausted or deposit log full). */
long h_replay(const double *q, const double *rn, long n, int *dir, double *de,
              long d_capacity, long *ndep) {
    stack.np = 0;
    stack.x[0] = q[0]; stack.y[0] = q[1]; stack.z[0] = q[2];
    stack.u[0] = q[3]; stack.v[0] = q[4]; stack.w[0] = q[5];
    stack.e[0] = q[6]; stack.wt[0] = q[7]; stack.ir[0] = (int)q[8]; stack.iq[0] = (int)q[9];
    stack.dnear[0] = q[10];
    rn_buf = (double *)rn; rn_cap = n; rn_pos = 0; rn_overflow = 0;
    dep_ir = dir; dep_e = de; dep_cap = d_capacity; dep_pos = 0; dep_overflow = 0;
    rng_mode = 2;
    dep_log_on = 1;
    shower();
    rng_mode = 0;
    dep_log_on = 0;
    *ndep = dep_pos;
    return (rn_overflow || dep_overflow) ? -1 : rn_pos;
}

void h_trace_draws(const char **sites, long cap) {
    draw_site = sites;
    draw_cap = cap;
}

/* h_replay with the count of random numbers drawn before each deposit. */
long h_replay_traced(const double *q, const double *rn, long n, int *dir, double *de, long *rnpos,
                     long d_capacity, long *ndep) {
    dep_rnpos = rnpos;
    long r = h_replay(q, rn, n, dir, de, d_capacity, ndep);
    dep_rnpos = NULL;
    return r;
}

/* Sampler entry points on a hand-set stack top with a scripted stream.
   which: 0 compton, 1 photo, 2 pair, 3 rayleigh, 4 moller, 5 bhabha,
   6 brems, 7 annih, 8 rannih.  q[11] is the particle (x,y,z,u,v,w,e,wt,ir,
   iq,dnear); out receives up to 4 particles of 11 doubles, top of stack
   last.  Returns the number of particles on the stack after the call. */
int h_sampler(int which, const double *q, const double *rn, long n, long *used, double *out) {
    stack.np = 0;
    stack.x[0] = q[0]; stack.y[0] = q[1]; stack.z[0] = q[2];
    stack.u[0] = q[3]; stack.v[0] = q[4]; stack.w[0] = q[5];
    stack.e[0] = q[6]; stack.wt[0] = q[7]; stack.ir[0] = (int)q[8]; stack.iq[0] = (int)q[9];
    stack.dnear[0] = q[10];
    rn_buf = (double *)rn; rn_cap = n; rn_pos = 0; rn_overflow = 0;
    rng_mode = 2;
    int imed = region.med[stack.ir[0]];
    double eig = stack.e[0], gle = log(eig);
    int lgle = 0;
    switch (which) {
    case 0: compton(); break;
    case 1: photo(); break;
    case 2: pair(imed); break;
    case 3:
        lgle = pwlfInterval(imed, gle, photon_data.ge1, photon_data.ge0) - 1;
        rayleigh(imed, eig, gle, lgle);
        break;
    case 4: moller(); break;
    case 5: bhabha(); break;
    case 6: brems(); break;
    case 7: annih(); break;
    case 8: rannih(); break;
    default: break;
    }
    rng_mode = 0;
    *used = rn_overflow ? -1 : rn_pos;
    int np = stack.np;
    for (int i = 0; i <= np && i < 4; i++) {
        double *o = out + 11 * i;
        o[0] = stack.x[i]; o[1] = stack.y[i]; o[2] = stack.z[i];
        o[3] = stack.u[i]; o[4] = stack.v[i]; o[5] = stack.w[i];
        o[6] = stack.e[i]; o[7] = stack.wt[i]; o[8] = stack.ir[i]; o[9] = stack.iq[i];
        o[10] = stack.dnear[i];
    }
    return np + 1;
}

/* Reference msdist on a hand-set electron with a scripted stream;
   returns ustep, fills fin[6] = x,y,z,u,v,w final. */
double h_msdist(const double *q, double de, double tustep, const double *rn, long n,
                long *used, double *fin) {
    stack.np = 0;
    stack.x[0] = q[0]; stack.y[0] = q[1]; stack.z[0] = q[2];
    stack.u[0] = q[3]; stack.v[0] = q[4]; stack.w[0] = q[5];
    stack.e[0] = q[6]; stack.wt[0] = q[7]; stack.ir[0] = (int)q[8]; stack.iq[0] = (int)q[9];
    rn_buf = (double *)rn; rn_cap = n; rn_pos = 0; rn_overflow = 0;
    rng_mode = 2;
    int irl = stack.ir[0];
    int imed = region.med[irl];
    double ustep = msdist(imed, stack.iq[0], region.rhof[irl], de, tustep, stack.e[0] - RM,
                          &fin[0], &fin[1], &fin[2], &fin[3], &fin[4], &fin[5]);
    rng_mode = 0;
    *used = rn_overflow ? -1 : rn_pos;
    return ustep;
}
