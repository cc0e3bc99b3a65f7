/*
 * omc_matrad_gpu: matRad's dose-influence MEX entry on the B200 engine.
 *
 *   [D, V] = omc_matrad_gpu(cubeRho, cubeMatIx, mcGeo, mcSrc, mcOpt)
 *
 * A drop-in for ompMC's omc_matrad MEX (ucodes/omc_matrad/omc_matrad.c:1417
 * mexFunction): the same five inputs, the same argument checks and error
 * identifiers (parseInput, omc_matrad.c:137-353; initPhantom :362-420), and
 * the same outputs, a sparse nvox x nBixels matrix D of dose per history
 * (rows = MATLAB linear voxel index, entries above relDoseThreshold times
 * the column maximum; omc_matrad.c:1576-1720) and, with two outputs, the
 * variance of the mean V on the same pattern.  The transport runs through
 * the C ABI of include/omcgpu.h (omc_tables_build, omc_engine_create,
 * omc_run_beamlets); nothing here touches CUDA.
 *
 * mcOpt fields read: verbose, nHistories (default 1e4), nBatches (10),
 * nSplit, charge, global_ecut, global_pcut, randomSeeds, pegsFile,
 * pgs4formFile, dataFolder, outputFolder, spectrumFile, relDoseThreshold
 * (0.01), sourceGeometry ('point' | 'gaussian'), sourceGaussianWidth
 * (0.2123); and two of this engine's own: gpuDevice (0) and transport
 * ('event', the FP32-transport/FP64-tally form, default; 'plain', FP64).
 *
 * Build inside MATLAB (CUDA runtime linked statically into libomcgpu.so):
 *   mex -I<repo>/include omc_matrad_gpu.c -L<repo>/ompmc_b200 -lomcgpu
 */
#include "mex.h"

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "omcgpu.h"

#define ERR_ID "matRad:omc_matrad:Error"

/* A field of a 1x1 struct; a required field that is missing fails as the
 * reference's num2str of it does (omc_matrad.c:236-340). */
static const mxArray *field(const mxArray *s, const char *name, int required) {
    const mxArray *f = mxGetField(s, 0, name);
    if (!f && required) mexErrMsgIdAndTxt(ERR_ID, "Call to num2str not successful (%s missing)", name);
    return f;
}

static double num(const mxArray *s, const char *name, double def, int required) {
    const mxArray *f = field(s, name, required);
    return f ? mxGetScalar(f) : def;
}

/* String field into buf (NULL when absent and not required). */
static const char *str(const mxArray *s, const char *name, char *buf, size_t n, int required) {
    const mxArray *f = field(s, name, required);
    if (!f) return NULL;
    if (mxGetString(f, buf, (mwSize)n) != 0) mexErrMsgIdAndTxt(ERR_ID, "%s must be a string", name);
    return buf;
}

/* Engine-side failure: report the library's message under the entry's
 * error identifier. */
static void check(int rc, const omc_engine *e, const char *what) {
    if (rc == OMC_OK) return;
    const char *m = e ? omc_engine_last_error(e) : omc_last_error();
    mexErrMsgIdAndTxt(ERR_ID, "%s failed (%s): %s", what, omc_status_string(rc), m ? m : "");
}

/* The double vector of a field, at least n long. */
static const double *vec(const mxArray *s, const char *name, size_t n) {
    const mxArray *f = field(s, name, 1);
    if (!mxIsDouble(f) || mxGetNumberOfElements(f) < n)
        mexErrMsgIdAndTxt(ERR_ID, "%s must be a double array of at least %d elements", name, (int)n);
    return mxGetPr(f);
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    /* argument checks of mexFunction and parseInput, in the reference's order */
    if (nrhs != 5) mexErrMsgIdAndTxt("matRad:matRad_ompInterface:invalidNumInputs", "Two or three input arguments required.");
    if (nlhs > 2) mexErrMsgIdAndTxt("matRad:matRad_ompInterface:invalidNumOutputs", "Too many output arguments.");
    const mxArray *cubeRho = prhs[0], *cubeMatIx = prhs[1], *mcGeo = prhs[2], *mcSrc = prhs[3], *mcOpt = prhs[4];
    if (!mxIsDouble(cubeRho))
        mexErrMsgIdAndTxt("matRad:matRad_ompInterface:inputNotDouble", "Input argument must be of type double.");
    if (mxGetNumberOfDimensions(cubeRho) != 3)
        mexErrMsgIdAndTxt("matRad:matRad_ompInterface:inputNot3D", "Input argument 1 must be a three-dimensional cube\n");
    if (!mxIsInt32(cubeMatIx))
        mexErrMsgIdAndTxt("matRad:matRad_ompInterface:inputNotInt32", "The density cube must be a 32 bit integer array!");
    if (!mxIsStruct(mcGeo)) mexErrMsgIdAndTxt("MATLAB:phonebook:inputNotStruct", "Input 3 must be a mcGeo Structure.");
    if (!mxIsStruct(mcSrc)) mexErrMsgIdAndTxt("MATLAB:phonebook:inputNotStruct", "Input 4 must be a mcSrc Structure.");

    /* options */
    int verbose = (int)num(mcOpt, "verbose", 0, 0);
    double nhist = num(mcOpt, "nHistories", 1e4, 0);
    int nbatch = (int)num(mcOpt, "nBatches", 10, 0);
    int nsplit = (int)num(mcOpt, "nSplit", 1, 1);
    if (nsplit < 1 || nsplit > OMC_MAX_NSPLIT) mexErrMsgIdAndTxt(ERR_ID, "nSplit must be between 1 and %d", OMC_MAX_NSPLIT);
    int charge = (int)num(mcOpt, "charge", 0, 1);
    double ecut = num(mcOpt, "global_ecut", 0, 1);
    double pcut = num(mcOpt, "global_pcut", 0, 1);
    const mxArray *fs = field(mcOpt, "randomSeeds", 1);
    const double *sv = mxGetPr(fs);
    uint64_t seed = ((uint64_t)(uint32_t)sv[0] << 32) |
                    (mxGetNumberOfElements(fs) > 1 ? (uint64_t)(uint32_t)sv[1] : 0u);
    char pegs[4096], pgs4[4096], data[4096], outdir[4096], spec[4096], geo[64], transport[64];
    str(mcOpt, "pegsFile", pegs, sizeof pegs, 1);
    str(mcOpt, "pgs4formFile", pgs4, sizeof pgs4, 1);
    str(mcOpt, "dataFolder", data, sizeof data, 1);
    str(mcOpt, "outputFolder", outdir, sizeof outdir, 1);
    if (!str(mcOpt, "spectrumFile", spec, sizeof spec, 0)) strcpy(spec, "./spectra/mohan6.spectrum");
    double rel = num(mcOpt, "relDoseThreshold", 0.01, 0);
    if (!str(mcOpt, "sourceGeometry", geo, sizeof geo, 0)) strcpy(geo, "point");
    double gwidth = num(mcOpt, "sourceGaussianWidth", 0.2123, 0);
    int device = (int)num(mcOpt, "gpuDevice", 0, 0);
    if (!str(mcOpt, "transport", transport, sizeof transport, 0)) strcpy(transport, "event");
    int mode = strcmp(transport, "plain") == 0 ? OMC_PLAIN_FP64 : OMC_EVENT_FP32;
    if (verbose) mexPrintf("omc_matrad_gpu: %s transport on GPU %d\n", mode == OMC_PLAIN_FP64 ? "plain FP64" : "event FP32", device);

    /* geometry (initPhantom, omc_matrad.c:362-420) */
    const mxArray *mat = mxGetField(mcGeo, 0, "material");
    if (!mat) mexErrMsgIdAndTxt(ERR_ID, "No materials specified!");
    int nmed = (int)mxGetDimensions(mat)[0];
    if (nmed < 1 || nmed > 9) mexErrMsgIdAndTxt(ERR_ID, "No materials specified!");
    char names[9][128];
    const char *media[9];
    for (int i = 0; i < nmed; i++) {
        mwIndex subs[2] = {(mwIndex)i, 0};
        const mxArray *c = mxGetCell(mat, mxCalcSingleSubscript(mat, 2, subs));
        if (!c) mexErrMsgIdAndTxt(ERR_ID, "Material could not be read!");
        char *s = mxArrayToString(c);
        if (!s) mexErrMsgIdAndTxt(ERR_ID, "Material string could not be read!");
        strncpy(names[i], s, sizeof names[i] - 1);
        names[i][sizeof names[i] - 1] = 0;
        media[i] = names[i];
    }
    const mwSize *dim = mxGetDimensions(cubeRho);
    int nx = (int)dim[0], ny = (int)dim[1], nz = (int)dim[2];
    const mwSize *mdim = mxGetDimensions(cubeMatIx);
    if (mxGetNumberOfDimensions(cubeMatIx) != 3 || (int)mdim[0] != nx || (int)mdim[1] != ny || (int)mdim[2] != nz)
        mexErrMsgIdAndTxt(ERR_ID, "cubeMatIx and cubeRho differ in shape");
    omc_phantom ph;
    ph.nx = nx;
    ph.ny = ny;
    ph.nz = nz;
    ph.xb = vec(mcGeo, "xBounds", (size_t)nx + 1);
    ph.yb = vec(mcGeo, "yBounds", (size_t)ny + 1);
    ph.zb = vec(mcGeo, "zBounds", (size_t)nz + 1);
    ph.rho = mxGetPr(cubeRho);
    ph.med = (const int32_t *)mxGetPr(cubeMatIx);  /* x fastest, media from 1, as the reference reads it */
    size_t nvox = (size_t)nx * ny * nz;
    for (size_t v = 0; v < nvox; v++)
        if (ph.med[v] < 1 || ph.med[v] > nmed) mexErrMsgIdAndTxt(ERR_ID, "material index outside 1..number of materials");

    /* beamlets (initSource, omc_matrad.c:618-832) */
    int nbix = (int)num(mcSrc, "nBixels", 0, 1);
    const double *ib = vec(mcSrc, "iBeam", (size_t)nbix);
    int32_t *ibeam = (int32_t *)mxCalloc((size_t)nbix + 1, sizeof(int32_t));
    int nbeams = 0;
    for (int i = 0; i < nbix; i++) {
        ibeam[i] = (int32_t)ib[i] - 1;
        if (ibeam[i] < 0) mexErrMsgIdAndTxt(ERR_ID, "iBeam / source position arrays are inconsistent");
        if (ibeam[i] + 1 > nbeams) nbeams = ibeam[i] + 1;
    }
    const char *sn[3] = {"xSource", "ySource", "zSource"};
    const char *bn[3][3] = {{"xCorner", "yCorner", "zCorner"}, {"xSide1", "ySide1", "zSide1"},
                            {"xSide2", "ySide2", "zSide2"}};
    double *src = (double *)mxCalloc((size_t)nbeams * 3 + 1, sizeof(double));
    double *pts[3];
    for (int c = 0; c < 3; c++) {
        const double *a = vec(mcSrc, sn[c], (size_t)nbeams);
        for (int i = 0; i < nbeams; i++) src[3 * i + c] = a[i];
    }
    for (int k = 0; k < 3; k++) {
        pts[k] = (double *)mxCalloc((size_t)nbix * 3 + 1, sizeof(double));
        for (int c = 0; c < 3; c++) {
            const double *a = vec(mcSrc, bn[k][c], (size_t)nbix);
            for (int i = 0; i < nbix; i++) pts[k][3 * i + c] = a[i];
        }
    }
    FILE *sf = fopen(spec, "r");
    if (!sf) mexErrMsgIdAndTxt(ERR_ID, "Unable to open file: %s", spec);
    fclose(sf);
    double *cdf1 = (double *)mxCalloc(1000, sizeof(double)), *cdf2 = (double *)mxCalloc(1000, sizeof(double));
    int ncdf = 0;
    check(omc_spectrum_load(spec, cdf1, cdf2, &ncdf), NULL, "spectrum");
    omc_beamlets bl;
    memset(&bl, 0, sizeof bl);
    bl.energy.charge = charge;
    bl.energy.mono_energy = 0.1;
    bl.energy.n = ncdf;
    bl.energy.cdf1 = cdf1;
    bl.energy.cdf2 = cdf2;
    bl.nbeams = nbeams;
    bl.nbixels = nbix;
    bl.ibeam = ibeam;
    bl.src = src;
    bl.corner = pts[0];
    bl.side1 = pts[1];
    bl.side2 = pts[2];
    bl.gaussian = strcmp(geo, "gaussian") == 0;
    bl.gauss_width = gwidth;

    /* tables, engine, run */
    omc_tables *tab = NULL;
    check(omc_tables_build(pegs, pgs4, data, media, nmed, &tab), NULL, "omc_tables_build");
    omc_options opt;
    omc_options_default(&opt);
    opt.ecut = ecut;
    opt.pcut = pcut;
    opt.device = device;
    opt.nsplit = nsplit;
    omc_engine *eng = NULL;
    int rc = omc_engine_create(tab, &ph, &opt, &eng);
    if (rc) {
        omc_tables_free(tab);
        check(rc, NULL, "omc_engine_create");
    }
    int64_t cap = (int64_t)(nvox * (size_t)nbix / 20 + 1024);
    int64_t *colptr = (int64_t *)mxCalloc((size_t)nbix + 1, sizeof(int64_t));
    int32_t *rows = NULL;
    double *vals = NULL, *var = NULL;
    int64_t nnz = 0;
    for (int attempt = 0; attempt < 3; attempt++) {
        rows = (int32_t *)mxCalloc((size_t)cap, sizeof(int32_t));
        vals = (double *)mxCalloc((size_t)cap, sizeof(double));
        var = (double *)mxCalloc((size_t)cap, sizeof(double));
        rc = omc_run_beamlets(eng, &bl, (int64_t)nhist, nbatch, rel, seed, mode, colptr, rows, vals, var, cap, &nnz,
                              NULL);
        if (rc != OMC_E_RANGE || nnz <= cap) break;
        mxFree(rows);
        mxFree(vals);
        mxFree(var);
        cap = nnz;
    }
    if (rc) {
        char msg[512];
        snprintf(msg, sizeof msg, "%s", omc_engine_last_error(eng));
        omc_engine_destroy(eng);
        omc_tables_free(tab);
        mexErrMsgIdAndTxt(ERR_ID, "omc_run_beamlets failed (%s): %s", omc_status_string(rc), msg);
    }
    omc_engine_destroy(eng);
    omc_tables_free(tab);

    /* outputs: sparse D (and V) in MATLAB's CSC layout */
    for (int k = 0; k < (nlhs > 1 ? 2 : 1); k++) {
        mxArray *m = mxCreateSparse((mwSize)nvox, (mwSize)nbix, (mwSize)(nnz > 0 ? nnz : 1), mxREAL);
        double *pr = mxGetPr(m);
        mwIndex *ir = mxGetIr(m), *jc = mxGetJc(m);
        const double *src_vals = k == 0 ? vals : var;
        for (int64_t i = 0; i < nnz; i++) {
            pr[i] = src_vals[i];
            ir[i] = (mwIndex)rows[i];
        }
        for (int j = 0; j <= nbix; j++) jc[j] = (mwIndex)colptr[j];
        plhs[k] = m;
    }
    if (verbose) mexPrintf("omc_matrad_gpu: %d beamlets, %lld nonzeros\n", nbix, (long long)nnz);
    mxFree(rows);
    mxFree(vals);
    mxFree(var);
    mxFree(colptr);
    mxFree(cdf1);
    mxFree(cdf2);
    mxFree(src);
    for (int k = 0; k < 3; k++) mxFree(pts[k]);
    mxFree(ibeam);
}
