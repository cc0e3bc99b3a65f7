/*
 * omcgpu — C ABI of the B200 dose engine (coupled photon/electron
 * condensed-history Monte Carlo on voxel phantoms).
 *
 * Every entry point returns an int status: OMC_OK (0) or a negative
 * OMC_E_* code; the message of the last failure of an engine is available
 * from omc_engine_last_error(), and process-wide failures from
 * omc_last_error().  Nothing in the library calls exit() or longjmp()
 * (ompMC exits the process on any error, e.g. ompmc.c:231-234).
 *
 * Arrays are plain C arrays owned by the caller; sizes are passed
 * explicitly.  Voxel arrays are x-fastest: v = i + j*nx + k*nx*ny, which is
 * ompMC's region number minus one (omc_dosxyz.c:124-128).
 *
 * Threading: one host thread drives an engine at a time, except through a
 * server: the omc_server_* calls of one server may come from any number of
 * host threads (they serialise on the server's mutex), so producers can
 * submit requests while another thread steps the server and collects
 * results.
 */
#ifndef OMCGPU_H
#define OMCGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define OMC_OK 0
#define OMC_E_ARG -1      /* invalid argument */
#define OMC_E_IO -2       /* file cannot be opened */
#define OMC_E_FORMAT -3   /* malformed file or data */
#define OMC_E_MEDIA -4    /* medium missing from the PEGS4 file */
#define OMC_E_RANGE -5    /* input outside a supported range */
#define OMC_E_CUDA -10    /* CUDA runtime failure (no device, launch error) */
#define OMC_E_NOMEM -11   /* device allocation failed / over budget */
#define OMC_E_DEVICE -12  /* a kernel raised an error flag (see last error) */
#define OMC_E_BUSY -13    /* serving queue full */
#define OMC_E_NOTREADY -14 /* request still running */

const char *omc_status_string(int status);
const char *omc_last_error(void);
int omc_version(void);

/* ------------------------------------------------------------ tables
 * Builds every physics table for the named media from a PEGS4 file, the
 * pgs4form file and a data folder holding xcom_{photo,rayleigh,pair,
 * triplet}.data, msnew.data and spinms.data.  Replaces ompMC's
 * initMediaData() (ompmc.c:5468-5503), which reads the same files through
 * the `.inp` keys `pegs file`, `pgs4form file` and `data folder`.
 * Host-only: needs no GPU. */
typedef struct omc_tables omc_tables;
int omc_tables_build(const char *pegs_file, const char *pgs4form_file, const char *data_folder,
                     const char *const *media, int nmed, omc_tables **out);
void omc_tables_free(omc_tables *t);
/* Read access to a table by ompMC's name (e.g. "gmfp0", "spin_rej",
 * "range_ep"; the struct fields of ompmc.h:107-406).  *is_int tells whether
 * *data points at int32 or double. */
int omc_tables_get(const omc_tables *t, const char *name, const void **data, int64_t *n, int *is_int);
int omc_tables_nmed(const omc_tables *t);

/* ------------------------------------------------------------ phantom
 * Rectilinear voxel phantom (omc_dosxyz.c:47-60, omc_matrad.c:364-453).
 * med: 1-based medium index per voxel (0 = vacuum); rho: g/cm^3. */
typedef struct {
    int nx, ny, nz;
    const double *xb, *yb, *zb; /* nx+1, ny+1, nz+1 boundaries (cm) */
    const int32_t *med;         /* nx*ny*nz */
    const double *rho;          /* nx*ny*nz */
} omc_phantom;

/* ------------------------------------------------------------ engine */
#define OMC_PLAIN_FP64 0   /* history-based, one thread per history, FP64 */
#define OMC_EVENT_FP32 1   /* event-based queues, FP32 transport, FP64 tallies */
#define OMC_EVENT_FP64 2   /* the same event-based form with FP64 transport
                              (omc_run_beam only; no photon splitting):
                              separates the event form's gain from FP32's */
#define OMC_MAX_NSPLIT 64  /* largest photon splitting factor (omc_options.nsplit) */

typedef struct {
    double ecut;          /* global ecut, total energy (MeV) ("global ecut") */
    double pcut;          /* global pcut (MeV) ("global pcut") */
    int device;           /* CUDA device ordinal */
    int ref_compat;       /* 1: reproduce ompMC's sampling quirks (default) */
    int64_t queue_capacity; /* event form: particles per queue (0 = default) */
    int block;            /* threads per block (0 = default; event form: a
                             multiple of 32, at most 256) */
    int nsplit;           /* photon splitting factor, 1 (off) to OMC_MAX_NSPLIT;
                             each photon interaction is sampled nsplit times at
                             weight 1/nsplit, photons from electrons are played
                             Russian roulette (ompmc.c:1867-2139, 4169-4182) */
    int profile;          /* 1: event form launches cycles one by one and times
                             every kernel (see omc_profile_last) */
    int electron_tsteps;  /* event form: tstep-loop iterations an electron runs
                             per launch before it is re-queued (0 = default 1) */
    int64_t inflight;     /* event form: particles kept in flight (0 = default) */
    int tail_boost;       /* event form: largest factor by which event budgets
                             grow as the queues drain (0 = default 32, 1 = fixed
                             budgets); results do not depend on it */
    double electron_split; /* event form: electrons above this kinetic energy
                             (MeV) are queued apart from the others so that
                             warps see particles of one kind (0 = one group,
                             the default); results do not depend on it */
    int electron_chsteps; /* event form: condensed-history steps after which an
                             electron's distance to its next discrete
                             interaction is drawn afresh (memoryless, so the
                             sampled physics is the same; default 3; 0 = the
                             reference's restart after every step, which
                             also costs a zero-length step each time) */
    int electron_interact_kernel; /* event form: 1 (default) = electrons'
                             discrete interactions are sampled in a kernel of
                             their own after the transport kernel (0 = in
                             place); results do not depend on it */
    int photon_woodcock;  /* event form: 1 (default) = photons are tracked by
                             delta (Woodcock) tracking against the largest
                             attenuation in the phantom instead of voxel by
                             voxel, when the grid is uniform (same sampled
                             distribution) */
    int64_t drain_particles; /* event form: once every history is injected and
                             at most this many particles are left, they are
                             run to the end of their sub-histories in one
                             launch instead of further cycles (0 = default,
                             half of the drain kernel's resident threads;
                             -1 = never);
                             results do not depend on it */
} omc_options;

void omc_options_default(omc_options *o);

typedef struct omc_engine omc_engine;
/* Uploads tables and phantom once; they stay resident across runs. */
int omc_engine_create(const omc_tables *t, const omc_phantom *ph, const omc_options *o, omc_engine **out);
int omc_engine_destroy(omc_engine *e);
/* Event-form tuning parameters of a live engine (the options of the same
 * names; a value <= 0 keeps the current one, for electron_split and
 * electron_chsteps a value < 0, for drain_particles -2).  Dose does not
 * depend on them (up to the summation order of the FP64 tallies) except
 * electron_chsteps, on which its distribution does not depend; the
 * autotuner (ompmc_b200/autotune.py) sweeps them. */
int omc_event_params(omc_engine *e, int electron_tsteps, int tail_boost, int64_t inflight, int block,
                     double electron_split, int electron_chsteps, int64_t drain_particles);
const char *omc_engine_last_error(const omc_engine *e);

/* Per-kernel profile of the last event-form omc_run_beam made with
 * options.profile = 1.  out (n >= 28) receives, for kernel k = 0 source,
 * 1 photon transport, 2 electron transport, 3 cycle planning, the values
 * out[k*7 + j]: j = 0 launches, 1 device seconds, 2 particles processed,
 * 3 transport steps (photon voxel steps, electron CH/BCA steps),
 * 4 voxel-boundary crossings, 5 energy deposits, 6 FP64 tally atomics
 * (deposits into one voxel in a row are summed first). */
int omc_profile_last(const omc_engine *e, double *out, int n);

/* Per-cycle trace of the last profiled event-form beam run: for cycle c,
 * out[6c .. 6c+5] = histories injected, particles in the photon queue
 * (injected primaries counted there) and in the electron queue at the start
 * of the transport kernels, and the source, photon and electron kernel times
 * in ms.  Copies at most max_cycles rows; returns the number of cycles
 * of that run (0 when none was profiled). */
int omc_profile_trace(const omc_engine *e, double *out, int max_cycles);

/* The drain of the last profiled event-form beam run (no reference
 * counterpart; instrumentation of this engine's end-of-run kernel): out
 * (n >= 5) = its device ms, the particles it started from, and the
 * largest sub-history one of its threads ran: events, events of the
 * particle it started from, transport steps.  Zeros when the run had no
 * drain. */
int omc_profile_drain(const omc_engine *e, double *out, int n);

/* ------------------------------------------------------------ sources */
/* Energy distribution: a spectrum inverse CDF (cdf1/cdf2 of length n,
 * omc_dosxyz.c:474-494) or a mono-energetic source (n = 0). */
typedef struct {
    int charge;             /* 0 photons, -1 electrons, +1 positrons */
    double mono_energy;     /* MeV kinetic, when n == 0 */
    int n;                  /* inverse-CDF size (ompMC: INVDIM = 1000) */
    const double *cdf1, *cdf2;
} omc_energy;

/* Reads a `.spectrum` file into an inverse CDF of 1000 points
 * (omc_dosxyz.c:368-510).  cdf1 and cdf2 must hold 1000 doubles. */
int omc_spectrum_load(const char *path, double *cdf1, double *cdf2, int *n);

/* Collimated point source on the z axis at distance ssd above the z = zmin
 * face (omc_dosxyz.c:337-632 and initHistory :964-1068). */
typedef struct {
    omc_energy energy;
    double ssd;
    double xinl, xinu, yinl, yinu; /* collimator rectangle on the surface */
} omc_beam;

/* matRad beamlets (omc_matrad.c:618-832, initHistory(ibeamlet) :1177-1413):
 * a point on the bixel parallelogram corner + r1*side1 + r2*side2, aimed
 * from the beam's source point (or a Gaussian spot of width gauss_width in
 * the bixel plane) and traced to the phantom surface. */
typedef struct {
    omc_energy energy;
    int nbeams, nbixels;
    const int32_t *ibeam;       /* nbixels, 0-based beam of each bixel */
    const double *src;          /* nbeams*3 */
    const double *corner;       /* nbixels*3 */
    const double *side1;        /* nbixels*3 */
    const double *side2;        /* nbixels*3 */
    int gaussian;               /* 0 point source, 1 Gaussian spot */
    double gauss_width;         /* cm */
} omc_beamlets;

/* --------------------------------------------------- dose runs (dosxyz)
 * Runs ncase histories (rounded down to nbatch*(ncase/nbatch), as
 * omc_dosxyz.c:1222-1229) of the beam in `mode`, tallying energy per batch,
 * and returns dose in Gy per incident particle and the batch-method
 * relative uncertainty per voxel (accumulateResults, omc_dosxyz.c:719-799,
 * voxels with rho < 0.044 zeroed).  dose/unc: nvox doubles (may be NULL).
 * stats (may be NULL) receives [0] histories run, [1] device seconds of the
 * transport, [2] kernel launches, [3] deposited energy (MeV), [4] source
 * energy (MeV), [5] error flags.  The engine keeps the run's device
 * buffers (tallies, sums, outputs; event form: nbatch*nvox batch tallies)
 * between calls, so repeated runs allocate nothing; they are released
 * with the engine. */
int omc_run_beam(omc_engine *e, const omc_beam *b, int64_t ncase, int nbatch, uint64_t seed, int mode,
                 double *dose, double *unc, double *stats);

/* ------------------------------------- fixed-scratch beam run (no alloc)
 * omc_run_beam in the plain FP64 form for callers that must not allocate
 * device memory while they run it: cudaMalloc/cudaFree synchronise the
 * device and take unbounded time, which a latency-bound caller (a plan
 * optimiser evaluating dose in its loop) cannot afford, and a host whose
 * GPU memory is owned by its own fixed-budget pool allocator may see an
 * extra allocation fail.  Create the engine at start-up, then call this.
 * It has no counterpart in the reference.
 *
 * All scratch (batch tallies, sums, outputs before download, spectrum)
 * lives in one file-scope device array sized for OMC_NOALLOC_MAX_VOXELS
 * voxels (about 10 MB), held by every GPU that loads the library until the
 * process exits.  Phantoms above that size are rejected with OMC_E_RANGE.
 * The first call on a device is a warm-up to make at start-up: it loads the
 * library's kernels on that device (lazy module loading), which may
 * allocate, and looks the array's address up (cudaGetSymbolAddress); make
 * it before any stream capture.  Later calls allocate nothing.  The address
 * is looked up again when the device's context has changed (after
 * cudaDeviceReset, for instance). 
 * Every call shares the array and clears it at its start: calls that
 * overlap on the GPU (other threads, other engines on the same device)
 * race.  Arguments and results are those of omc_run_beam with mode
 * OMC_PLAIN_FP64; stats[1] is host wall time of the run.  Engines with
 * photon splitting (nsplit > 1) are rejected with OMC_E_RANGE: their
 * kernels need a deeper per-thread stack, which the driver may grow on
 * first launch. */
#define OMC_NOALLOC_MAX_VOXELS 262144
int omc_run_beam_noalloc(omc_engine *e, const omc_beam *b, int64_t ncase, int nbatch, uint64_t seed, double *dose,
                         double *unc, double *stats);

/* ------------------------------------------- dose influence (matRad)
 * One sparse column per beamlet, as the matRad MEX entry builds them
 * (omc_matrad.c:1576-1720): per beamlet, nhist histories in nbatch
 * batches, dose in Gy per history (accumEndep divides by the histories of
 * a batch, omc_matrad.c:897-918), entries above rel_threshold * column
 * maximum kept, rows = voxel index.  Variance of the mean in var (may be
 * NULL).  The CSC arrays are caller-owned: colptr has nbixels+1 entries;
 * rows/vals/var have room for cap entries; *nnz receives the total, and
 * OMC_E_RANGE is returned (with *nnz the size needed) when cap is short. */
int omc_run_beamlets(omc_engine *e, const omc_beamlets *b, int64_t nhist, int nbatch, double rel_threshold,
                     uint64_t seed, int mode, int64_t *colptr, int32_t *rows, double *vals, double *var,
                     int64_t cap, int64_t *nnz, double *stats);

/* ------------------------------------------------------------ serving
 * Continuous batching: beam and beamlet requests of any history count are
 * admitted while device memory for their tallies is within `mem_budget`
 * bytes (0: half the free memory, at most 32 GB; each request holds
 * 10 * nvox * 8 bytes of batch tallies), at most `max_requests` (<= 256,
 * 0 = 256) at a time; all admitted requests share the same particle
 * queues, and requests beyond the budget wait and are admitted first come
 * first served as earlier ones finish.  omc_server_* replace the
 * sequential beamlet loop of omc_matrad.c:1576.  OMC_E_NOMEM when the
 * budget holds no request.  Thread-safe: every call on a server holds its
 * mutex, so submissions from other threads wait for a step in progress
 * (at most a few transport cycles). */
typedef struct omc_server omc_server;
int omc_server_create(omc_engine *e, int64_t mem_budget, int max_requests, uint64_t seed, omc_server **out);
int omc_server_destroy(omc_server *s);
/* Submits one beamlet (index ibixel of b, which must outlive the request)
 * or one beam (its spectrum is copied); nbatch 2..10.  A request's random
 * streams depend only on `seed` (0: derived from the server seed and the
 * request id), so its result is the same alone or among other requests.
 * Returns a request id >= 0 or a negative status. */
int omc_server_submit_beamlet(omc_server *s, const omc_beamlets *b, int ibixel, int64_t nhist, int nbatch,
                              double rel_threshold, uint64_t seed);
int omc_server_submit_beam(omc_server *s, const omc_beam *b, int64_t nhist, int nbatch, uint64_t seed);
/* Advances the device by up to `cycles` transport cycles, or, when nothing
 * is pending, every running request is fully injected and at most the
 * engine's drain_particles are left, by one drain launch that runs them to
 * the end; *active receives the requests still running. */
int omc_server_step(omc_server *s, int cycles, int *active);
/* Status of a request: OMC_OK when finished, OMC_E_NOTREADY while running. */
int omc_server_poll(omc_server *s, int id, double *latency_ms);
/* Sparse column of a finished beamlet request (rows, vals, var of
 * capacity cap; var may be NULL) or dense dose/unc of a beam request. */
int omc_server_result_sparse(omc_server *s, int id, int32_t *rows, double *vals, double *var, int64_t cap,
                             int64_t *nnz);
int omc_server_result_dense(omc_server *s, int id, double *dose, double *unc);
int omc_server_release(omc_server *s, int id);
/* Completion queue (no reference counterpart): copies into ids (capacity
 * cap) the requests that finished since the previous call, in the order
 * they finished, and removes them from the queue; *n receives the count. */
int omc_server_completed(omc_server *s, int *ids, int cap, int *n);
/* Device time of the server's stream between two marks (no reference
 * counterpart): stop = 0 records the start mark; stop = 1 records the end
 * mark, waits for it and returns the milliseconds between them in *ms. */
int omc_server_timer(omc_server *s, int stop, double *ms);
/* Counters of a server since its creation (no reference counterpart):
 * out (n >= 4) = transport cycles, drain launches, kernel launches
 * (cycles, drains, folds, finalisation and column extraction), requests
 * finished.  With options.profile = 1 the server launches its cycles one
 * by one with events around each kernel, and omc_profile_last reports the
 * per-kernel times and transport counters of everything it has run. */
int omc_server_stats(omc_server *s, double *out, int n);

/* ---------------------------------------------- drop-in CLI (dosxyz)
 * The whole omc_dosxyz program (omc_dosxyz.c:1072-1307): reads
 * `<inp_base>.inp` (same keys), runs and writes
 * `<output folder><out_name>.3ddose`.  mode selects the transport form. */
int omc_dosxyz_run(const char *inp_base, const char *out_name, int mode, int verbose);

/* ------------------------------------------------- validation hooks
 * Geometry: walks each ray (x,y,z,u,v,w,ir) straight through the phantom
 * with the FP64 device howfar (omc_dosxyz.c:187-297), recording ustep,
 * irnew and idisc of every call (up to cap per ray), like the photon
 * transport loop with an infinite interaction distance.  hownear_out
 * (nrays, may be NULL) receives hownear at each ray's start. */
int omc_trace_rays(omc_engine *e, const double *rays, int nrays, int cap, double *ustep, int32_t *irnew,
                   int32_t *idisc, int32_t *ncalls, double *hownear_out);
/* Transport: runs history h from primary prim[11*h] (x,y,z,u,v,w,e,wt,
 * ir,iq,dnear) with the FP64 physics on the scripted uniform stream
 * rn[rn_off[h] .. rn_off[h+1]), logging every deposit (region, energy)
 * into dep_ir/dep_e[h*dep_cap ...]; ndep[h] and nused[h] receive the
 * deposits and random numbers consumed. */
int omc_replay(omc_engine *e, const double *prim, int nhist, const double *rn, const int64_t *rn_off,
               int dep_cap, int32_t *dep_ir, double *dep_e, int32_t *ndep, int64_t *nused, uint32_t *flags);

/* Samplers: runs one FP64 interaction sampler per case on the scripted
 * uniform stream rn[rn_off[c] .. rn_off[c+1]) of case c, from the particle
 * q[11*c] (x,y,z,u,v,w,e,wt,ir,iq,dnear; e total energy).  which: 0 compton
 * (ompmc.c:1688-1801), 1 photo (:1804-1864), 2 pair (:1447-1685),
 * 3 rayleigh (:1120-1163), 4 moller (:4377-4453), 5 bhabha (:4456-4543),
 * 6 brems (:4188-4374), 7 annih (:4546-4663), 8 rannih (:4129-4185),
 * 9 msdist (:3805-3994, with de = extra[2c] and tustep = extra[2c+1]).
 * out[44*c ...] receives up to 4 particles of 11 doubles: the input particle
 * after the sampler, then what it pushed (msdist: ustep and the final
 * x,y,z,u,v,w); nout[c] their number, used[c] the random numbers drawn,
 * flags[c] device error bits (8: the stream ran out). */
int omc_kat(omc_engine *e, int which, const double *q, const double *extra, int n, const double *rn,
            const int64_t *rn_off, double *out, int32_t *nout, int64_t *used, uint32_t *flags);

/* Device allocations (cudaMalloc) the library has made in this process, all
 * engines and devices together; no reference counterpart.  Tests read it
 * around a call to show that the call allocated nothing. */
int64_t omc_device_allocations(void);

#ifdef __cplusplus
}
#endif
#endif /* OMCGPU_H */
