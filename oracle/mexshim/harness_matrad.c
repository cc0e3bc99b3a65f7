/*
 * Oracle harness for the matRad D_ij entry: the mx/mex shim functions and
 * hm_dij(), which builds matRad's five inputs from plain arrays and calls
 * the UNMODIFIED mexFunction of ucodes/omc_matrad/omc_matrad.c (compiled
 * single-threaded into oracle/_ref/libompmc_matrad_ref.so).  Test
 * infrastructure only.
 */
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "mex.h"

static jmp_buf g_jmp;
static char g_err[512];
static int g_quiet = 1;

/* Timing of the reference's beamlet loop: with hm_timing(1) the entry runs
 * with mcOpt.verbose = 2, which makes it create a waitbar before its
 * beamlet loop, update it after every batch and every beamlet and close it
 * after the loop (omc_matrad.c:1527-1530, 1594-1600, 1704-1712, 1720-1724);
 * the shim records the time and progress value of each of those calls. */
static int g_timing = 0;
#define WB_CAP 65536
static double g_wb_t[WB_CAP], g_wb_p[WB_CAP];
static int g_nwb = 0;

static double mono_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

void hm_timing(int on) { g_timing = on; }

/* Waitbar calls of the last hm_dij: time (s, monotonic) and progress
 * (-1 for the create and close calls); returns how many were recorded. */
int hm_waitbar_log(double *t, double *p, int cap) {
    int n = g_nwb < cap ? g_nwb : cap;
    for (int i = 0; i < n; i++) {
        t[i] = g_wb_t[i];
        p[i] = g_wb_p[i];
    }
    return n;
}

/* ----------------------------------------------------------- mx arrays */
static mxArray *mk(int cls) {
    mxArray *a = calloc(1, sizeof(mxArray));
    a->cls = cls;
    a->ndim = 2;
    a->dims[0] = a->dims[1] = 1;
    return a;
}

static mxArray *mk_double(const double *v, mwSize n0, mwSize n1, mwSize n2) {
    mxArray *a = mk(0);
    a->ndim = n2 > 1 ? 3 : 2;
    a->dims[0] = n0; a->dims[1] = n1; a->dims[2] = n2 > 0 ? n2 : 1;
    size_t n = n0 * n1 * (n2 > 0 ? n2 : 1);
    a->pr = malloc((n ? n : 1) * sizeof(double));
    if (v) memcpy(a->pr, v, n * sizeof(double));
    return a;
}

static mxArray *mk_int32(const int32_t *v, mwSize n0, mwSize n1, mwSize n2) {
    mxArray *a = mk(1);
    a->ndim = 3;
    a->dims[0] = n0; a->dims[1] = n1; a->dims[2] = n2;
    size_t n = n0 * n1 * n2;
    a->i32 = malloc(n * sizeof(int32_t));
    memcpy(a->i32, v, n * sizeof(int32_t));
    return a;
}

static mxArray *mk_struct(int nf) {
    mxArray *a = mk(3);
    a->fnames = calloc(nf, sizeof(char *));
    a->fvals = calloc(nf, sizeof(mxArray *));
    return a;
}

static void set_field(mxArray *s, const char *name, mxArray *v) {
    s->fnames[s->nfields] = name;
    s->fvals[s->nfields] = v;
    s->nfields++;
}

mxArray *mxCreateString(const char *str) {
    mxArray *a = mk(2);
    a->str = strdup(str ? str : "");
    a->dims[1] = strlen(a->str);
    return a;
}

mxArray *mxCreateDoubleScalar(double v) { return mk_double(&v, 1, 1, 0); }

void mxDestroyArray(mxArray *a) {
    if (!a) return;
    free(a->pr);
    free(a->i32);
    free(a->str);
    if (a->cls == 3)
        for (int i = 0; i < a->nfields; i++) mxDestroyArray(a->fvals[i]);
    free(a->fnames);
    free(a->fvals);
    if (a->cls == 4)
        for (mwSize i = 0; i < a->dims[0] * a->dims[1]; i++) mxDestroyArray(a->cells[i]);
    free(a->cells);
    free(a->ir);
    free(a->jc);
    free(a);
}

mxArray *mxGetField(const mxArray *a, mwIndex i, const char *name) {
    (void)i;
    if (!a || a->cls != 3) return NULL;
    for (int k = 0; k < a->nfields; k++)
        if (!strcmp(a->fnames[k], name)) return a->fvals[k];
    return NULL;
}

double *mxGetPr(const mxArray *a) {
    if (!a) return NULL;
    if (a->cls == 1) return (double *)a->i32;
    return a->pr;
}

double mxGetScalar(const mxArray *a) {
    if (!a) return 0.0;
    if (a->cls == 1) return (double)a->i32[0];
    if (a->cls == 0 || a->cls == 5) return a->pr ? a->pr[0] : 0.0;
    return 0.0;
}

char *mxArrayToString(const mxArray *a) {
    if (!a || a->cls != 2) return NULL;
    return strdup(a->str);
}

int mxGetString(const mxArray *a, char *buf, mwSize buflen) {
    if (!a || a->cls != 2 || buflen == 0) return 1;
    strncpy(buf, a->str, buflen - 1);
    buf[buflen - 1] = 0;
    return 0;
}

size_t mxGetNumberOfElements(const mxArray *a) {
    size_t n = 1;
    for (mwSize i = 0; i < a->ndim; i++) n *= a->dims[i];
    return n;
}

const mwSize *mxGetDimensions(const mxArray *a) { return a->dims; }
mwSize mxGetNumberOfDimensions(const mxArray *a) { return a->ndim; }

mwIndex mxCalcSingleSubscript(const mxArray *a, mwSize nsubs, const mwIndex *subs) {
    mwIndex idx = 0, mul = 1;
    for (mwSize k = 0; k < nsubs; k++) {
        idx += subs[k] * mul;
        mul *= a->dims[k];
    }
    return idx;
}

mxArray *mxGetCell(const mxArray *a, mwIndex i) { return (a && a->cls == 4) ? a->cells[i] : NULL; }
int mxIsDouble(const mxArray *a) { return a && a->cls == 0; }
int mxIsInt32(const mxArray *a) { return a && a->cls == 1; }
int mxIsStruct(const mxArray *a) { return a && a->cls == 3; }
int mxGetNumberOfFields(const mxArray *a) { return a ? a->nfields : 0; }

mxArray *mxCreateSparse(mwSize m, mwSize n, mwSize nzmax, int flag) {
    (void)flag;
    mxArray *a = mk(5);
    a->dims[0] = m;
    a->dims[1] = n;
    a->nzmax = nzmax ? nzmax : 1;
    a->pr = calloc(a->nzmax, sizeof(double));
    a->ir = calloc(a->nzmax, sizeof(mwIndex));
    a->jc = calloc(n + 1, sizeof(mwIndex));
    return a;
}

mwIndex *mxGetIr(const mxArray *a) { return a->ir; }
mwIndex *mxGetJc(const mxArray *a) { return a->jc; }
void mxSetPr(mxArray *a, double *p) { a->pr = p; }
void mxSetIr(mxArray *a, mwIndex *p) { a->ir = p; }
void mxSetNzmax(mxArray *a, mwSize n) { a->nzmax = n; }
void *mxRealloc(void *p, size_t n) { return realloc(p, n ? n : 1); }
void *mxCalloc(size_t n, size_t sz) { return calloc(n ? n : 1, sz ? sz : 1); }
void mxFree(void *p) { free(p); }

int mexPrintf(const char *fmt, ...) {
    if (g_quiet) return 0;
    va_list ap;
    va_start(ap, fmt);
    int r = vfprintf(stderr, fmt, ap);
    va_end(ap);
    return r;
}

void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    int k = snprintf(g_err, sizeof(g_err), "%s: ", id);
    vsnprintf(g_err + k, sizeof(g_err) - k, fmt, ap);
    va_end(ap);
    longjmp(g_jmp, 1);
}

/* num2str of a numeric array: values separated by two spaces, as MATLAB. */
int mexCallMATLAB(int nlhs, mxArray *plhs[], int nrhs, mxArray *prhs[], const char *name) {
    if (!strcmp(name, "num2str") && nrhs >= 1 && nlhs >= 1) {
        char buf[512] = {0};
        size_t n = prhs[0] ? mxGetNumberOfElements(prhs[0]) : 0;
        size_t off = 0;
        for (size_t i = 0; i < n && off < sizeof(buf) - 32; i++) {
            double v = prhs[0]->cls == 1 ? (double)prhs[0]->i32[i] : prhs[0]->pr[i];
            off += snprintf(buf + off, sizeof(buf) - off, i ? "  %.15g" : "%.15g", v);
        }
        plhs[0] = mxCreateString(buf);
        return 0;
    }
    if (g_timing && (!strcmp(name, "waitbar") || !strcmp(name, "close"))) {
        if (g_nwb < WB_CAP) {
            int upd = !strcmp(name, "waitbar") && nlhs == 0 && nrhs >= 1 && prhs[0] && prhs[0]->pr;
            g_wb_t[g_nwb] = mono_s();
            g_wb_p[g_nwb] = upd ? prhs[0]->pr[0] : -1.0;
            g_nwb++;
        }
        /* the create call's handle is destroyed by the caller after close */
        if (nlhs >= 1) plhs[0] = mxCreateDoubleScalar(1.0);
        return 0;
    }
    if (nlhs >= 1) plhs[0] = NULL;
    return 0;
}

/* ------------------------------------------------------------- harness */
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

const char *hm_last_error(void) { return g_err; }
void hm_verbose(int v) { g_quiet = !v; }

/*
 * One call of the matRad MEX entry.  Voxel arrays are x fastest (MATLAB
 * column-major [nx, ny, nz]).  Beam and bixel vectors as in matRad's mcSrc
 * (ibeam 1-based).  Outputs: the CSC arrays of D and V copied into
 * jc[nbix+1], ir/pr/var[cap]; returns nnz, or -1 on error (hm_last_error),
 * or -2 when cap is too small.
 */
long hm_dij(int nx, int ny, int nz, const double *rho, const int32_t *matix, int nmat, const char **materials,
            const double *xb, const double *yb, const double *zb, int nbix, int nbeams, const double *ibeam,
            const double *src /* nbeams*3 */, const double *corner, const double *side1, const double *side2,
            double nhist, double nbatch, double seed1, double seed2, double ecut, double pcut, double rel,
            const char *spectrum, const char *pegs, const char *pgs4form, const char *data_folder,
            const char *output_folder, int gaussian, double gwidth, long *jc, long *ir, double *pr, double *var,
            long cap) {
    mxArray *cubeRho = mk_double(rho, nx, ny, nz);
    mxArray *cubeMat = mk_int32(matix, nx, ny, nz);
    mxArray *geo = mk_struct(4);
    mxArray *mat = mk(4);
    mat->dims[0] = nmat;
    mat->dims[1] = 1;
    mat->cells = calloc(nmat, sizeof(mxArray *));
    for (int i = 0; i < nmat; i++) mat->cells[i] = mxCreateString(materials[i]);
    set_field(geo, "material", mat);
    set_field(geo, "xBounds", mk_double(xb, nx + 1, 1, 0));
    set_field(geo, "yBounds", mk_double(yb, ny + 1, 1, 0));
    set_field(geo, "zBounds", mk_double(zb, nz + 1, 1, 0));
    mxArray *msrc = mk_struct(14);
    double nb = nbix;
    set_field(msrc, "nBixels", mk_double(&nb, 1, 1, 0));
    set_field(msrc, "iBeam", mk_double(ibeam, nbix, 1, 0));
    double *tmp = malloc(sizeof(double) * (nbeams > nbix ? nbeams : nbix));
    const char *sn[3] = {"xSource", "ySource", "zSource"};
    for (int c = 0; c < 3; c++) {
        for (int i = 0; i < nbeams; i++) tmp[i] = src[3 * i + c];
        set_field(msrc, sn[c], mk_double(tmp, nbeams, 1, 0));
    }
    const char *cn[3][3] = {{"xCorner", "yCorner", "zCorner"}, {"xSide1", "ySide1", "zSide1"},
                            {"xSide2", "ySide2", "zSide2"}};
    const double *arr[3] = {corner, side1, side2};
    for (int k = 0; k < 3; k++)
        for (int c = 0; c < 3; c++) {
            for (int i = 0; i < nbix; i++) tmp[i] = arr[k][3 * i + c];
            set_field(msrc, cn[k][c], mk_double(tmp, nbix, 1, 0));
        }
    free(tmp);
    mxArray *opt = mk_struct(20);
    double zero = 0, one = 1, seeds[2] = {seed1, seed2};
    double verb = g_timing ? 2.0 : 0.0;
    set_field(opt, "verbose", mk_double(&verb, 1, 1, 0));
    set_field(opt, "nHistories", mk_double(&nhist, 1, 1, 0));
    set_field(opt, "nBatches", mk_double(&nbatch, 1, 1, 0));
    set_field(opt, "nSplit", mk_double(&one, 1, 1, 0));
    set_field(opt, "charge", mk_double(&zero, 1, 1, 0));
    set_field(opt, "global_ecut", mk_double(&ecut, 1, 1, 0));
    set_field(opt, "global_pcut", mk_double(&pcut, 1, 1, 0));
    set_field(opt, "randomSeeds", mk_double(seeds, 1, 2, 0));
    set_field(opt, "pegsFile", mxCreateString(pegs));
    set_field(opt, "pgs4formFile", mxCreateString(pgs4form));
    set_field(opt, "dataFolder", mxCreateString(data_folder));
    set_field(opt, "outputFolder", mxCreateString(output_folder));
    set_field(opt, "spectrumFile", mxCreateString(spectrum));
    set_field(opt, "relDoseThreshold", mk_double(&rel, 1, 1, 0));
    set_field(opt, "sourceGeometry", mxCreateString(gaussian ? "gaussian" : "point"));
    set_field(opt, "sourceGaussianWidth", mk_double(&gwidth, 1, 1, 0));
    const mxArray *in[5] = {cubeRho, cubeMat, geo, msrc, opt};
    mxArray *out[2] = {NULL, NULL};
    long nnz = -1;
    g_err[0] = 0;
    g_nwb = 0;
    if (setjmp(g_jmp) == 0) {
        mexFunction(2, out, 5, in);
        nnz = (long)out[0]->jc[nbix];
        if (nnz > cap) {
            nnz = -2;
        } else {
            for (int j = 0; j <= nbix; j++) jc[j] = (long)out[0]->jc[j];
            for (long k = 0; k < nnz; k++) {
                ir[k] = (long)out[0]->ir[k];
                pr[k] = out[0]->pr[k];
                var[k] = out[1]->pr[k];
            }
        }
    }
    mxDestroyArray(out[0]);
    mxDestroyArray(out[1]);
    for (int k = 0; k < 5; k++) mxDestroyArray((mxArray *)in[k]);
    return nnz;
}
