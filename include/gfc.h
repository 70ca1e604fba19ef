/*
 * gfc.h -- C ABI of the B200 Coulomb gauge fixer (libgfc.so).
 *
 * Plain pointers and sizes only; no CUDA or torch types cross this boundary, so
 * the library can be bound from C (the gauge_fix_coulomb CLI), ctypes, cgo or JNI.
 * Every entry point returns an int status (GFC_OK or a negative GFC_ERR_*), except
 * the ones that mirror a reference function returning something else; those keep
 * the reference's return convention and say so.
 *
 * Field layouts in HOST memory are the reference's (fields.h:33-43):
 *   links  U : [t][z][y][x][mu][row][col][re,im], mu = 0 (t), 1 (z), 2 (y), 3 (x)
 *   gauge  G : [t][z][y][x][row][col][re,im]
 * i.e. 4V (resp. V) 3x3 complex matrices, V = ns^3 * nt.  Device layouts are
 * private to the library (structure-of-arrays, checkerboard ordered).
 */
#ifndef GFC_H
#define GFC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------ */
#define GFC_OK            0
#define GFC_ERR_ARG      -10   /* bad argument (null pointer, bad size, ...)        */
#define GFC_ERR_NOMEM    -11   /* host or device allocation failed                  */
#define GFC_ERR_CUDA     -12   /* a CUDA runtime call failed                        */
#define GFC_ERR_GEOMETRY -13   /* lattice extents not supported                     */
#define GFC_ERR_IO       -14   /* file could not be opened / read / written         */
#define GFC_ERR_STATE    -15   /* call out of order (e.g. fix before upload)        */
#define GFC_ERR_BUSY     -16   /* serving queue full / no slot                       */
#define GFC_ERR_TIMEOUT  -17   /* a bounded wait ran out                             */
#define GFC_ERR_NUMERIC  -18   /* NaN or projection failure reported by a kernel    */

/* gaugefixOverrelaxation return codes (gauge_fixing.c:741-747) */
#define GFC_FIX_NOT_CONVERGED  -1
#define GFC_FIX_BAD_PARAMS     -2

/* ---- parameters (gauge_fixing.h:30-54) ---------------------------------------- */
typedef enum { GFC_PROXY_E2 = 0, GFC_PROXY_THETA = 1 } gfc_proxy;

/* Same members and meaning as ORGaugeFixingParameters; the proxy function pointer
 * becomes an enum because a host function pointer cannot run on the device.
 * omega_OR stays a float: the reference stores it as float (gauge_fixing.h:51) and
 * every update sees (double)(float)omega. */
typedef struct {
    double   tolerance;
    int      gfix_proxy;                     /* gfc_proxy */
    unsigned max_sweeps_to_fix;
    unsigned estimate_sweeps_to_gf_progress;
    unsigned sweeps_to_reunitarization;
    int      error;                          /* set by the parser on invalid values */
    float    omega_OR;
    unsigned hits;
} gfc_params;

/* Defaults of initParametersORDefault (gauge_fixing.c:72-84). */
void gfc_params_default(gfc_params *p);
/* validORGaugeFixingParametersQ (gauge_fixing.c:45-70): 1 if valid, 0 if not. */
int  gfc_params_valid(const gfc_params *p);
/* initORGaugeFixingParameters (gauge_fixing.c:144-244): same key:value parser,
 * same messages on stdout/stderr, accepts the parser's key names and the README /
 * print-label spellings (max_hits, estimate_sweeps_to_gfixprogress).  path == NULL
 * or " " means "no file": defaults.  Returns GFC_OK; p->error flags bad values. */
int  gfc_params_parse_file(const char *path, gfc_params *p);
/* printORGaugeFixingParameters (gauge_fixing.c:86-104), same text on stdout. */
void gfc_params_print(const gfc_params *p);

/* ---- run options (no counterpart in the reference: GPU execution choices) ---- */
typedef enum {
    GFC_PREC_FP64_EXACT = 0, /* FP64, reference arithmetic: bit-for-bit the reference update */
    GFC_PREC_FP64_FAST  = 1, /* FP64, direct SU(2) accumulation, FMA, two stored rows per matrix */
    GFC_PREC_MIXED      = 2, /* FP32 bulk sweeps (two rows), FP64 two-row refinement          */
    GFC_PREC_FP64_FULL  = 3  /* FP64 fast arithmetic on full 3x3 storage (plain FP64)          */
} gfc_precision;

typedef enum {
    GFC_STOP_REFERENCE = 0,  /* the reference check schedule (gauge_fixing.c:248-285,791-808) */
    GFC_STOP_EVERY     = 1   /* test the proxy after every half-sweep, stop at first <= tol    */
} gfc_stop_rule;

typedef struct {
    int    precision;         /* gfc_precision                                       */
    int    stop_rule;         /* gfc_stop_rule                                       */
    int    verbose;           /* print the reference's "Sweeps: ... residue" lines   */
    double switch_e2;         /* mixed: leave FP32 when e2 < switch_e2 (default 1e-9) */
    unsigned refine_reunit;   /* mixed: reunitarise every n FP64 half-sweeps (0: use params) */
    int    block_threads;     /* 0: library default / autotuned                      */
    int    dense_check;       /* GFC_STOP_EVERY on the fast paths: 0 (default) measures e2
                                 on one pair of half-sweeps per 32 while the measured rate
                                 says the tolerance is far, then after every half-sweep;
                                 1 measures after every half-sweep throughout            */
    int    warm_start;        /* 1: the resident G (gfc_ctx_upload_gt) is the starting
                                 transformation: the fix works on G U G^dagger and the G
                                 it returns includes it (loadGaugeTransf +
                                 applyGaugeTransformationU, fields_io.c:309-402,
                                 fields.c:375-435, then the fix); every precision (the
                                 mixed path re-gauges the uploaded links with G1 G0
                                 at its switch to FP64)                              */
    int    fp32_refresh;      /* mixed: every n FP32 half-sweeps fold the FP32 G into an
                                 FP64 G and rebuild the FP32 links from it as G U0
                                 G^dagger in FP64, so FP32 rounding does not accumulate
                                 in the links; the FP32 fields are then not
                                 reunitarised between rebuilds (0: off, FP32
                                 reunitarisation every min(reunit, 50) half-sweeps)   */
} gfc_options;

void gfc_options_default(gfc_options *o);

/* ---- run report ------------------------------------------------------------- */
typedef struct {
    int    status;            /* return value of the fix                           */
    int    sweeps;            /* half-sweeps performed                             */
    int    sweeps_fp32;       /* mixed: half-sweeps done in FP32                   */
    int    first_below_tol;   /* first half-sweep whose proxy was seen <= tol (-1 if not tracked) */
    double initial_residue;
    double final_residue;     /* proxy after the final reunitarisation             */
    double e2, theta, functional;
    double seconds_sweeps;    /* device time of the sweep loop                     */
    double seconds_total;     /* device time of the whole call                     */
    long long site_updates;   /* sum over half-sweeps of sites updated             */
    int    kernel_launches;   /* library kernels launched during the call          */
} gfc_report;

/* ---- synthetic configurations ------------------------------------------------ */
/* U = 4V matrices (4V*18 doubles, reference layout), built as
 * U_mu(x) = g(x) exp(i scale H_mu(x)) g(x+mu)^dagger with counter-based seeded
 * random numbers (see host/gfc_synth.c).  No counterpart in the reference (it
 * ships no inputs); used by the benchmarks and tests. */
int gfc_synth_config(int ns, int nt, uint64_t seed, double scale, double *U);

/* ---- host file access (fields_io.c) ------------------------------------------ */
#define GFC_FILE_CONFIG 0
#define GFC_FILE_GT     1
/* Exact-size read with the reference's messages and codes (loadConfig,
 * fields_io.c:216-305; loadGaugeTransf, fields_io.c:309-402):
 * 0, -1 cannot open, -2 short read, -3 (config) / -2 (gt) file too long. */
int gfc_read_exact(const char *path, void *buf, size_t bytes, int kind);
/* writeGaugeTransf / writeConfig file part (fields_io.c:405-565): 0, -1, -2 */
int gfc_write_all(const char *path, const void *buf, size_t bytes);
/* byteSwap (fields_io.c:42-96): reverse every word_bytes (1, 4 or 8) word; -1 otherwise */
int gfc_byteswap(void *buf, size_t word_bytes, size_t total_bytes);

/* ---- device contexts ------------------------------------------------------------ */
/* A context holds one lattice resident on one GPU: spatial links, temporal
 * links, gauge transformation, scratch.  Not thread-safe; one host thread per
 * context.  No counterpart in the reference, whose state is the global
 * lattice_param (geometry.h:113-119) plus caller-owned U and G arrays. */
typedef struct gfc_ctx gfc_ctx;
#define GFC_CTX_MIXED 1   /* also allocate the FP32 fields and the FP64 copy used by GFC_PREC_MIXED */

const char *gfc_last_error(void);
/* Architecture of the library's device code as loaded on `device`
 * (cudaFuncGetAttributes): binary_version 100 = sm_100 machine code, ptx_version =
 * the virtual architecture it was compiled for (100).  No counterpart in the
 * reference (it has no device code). */
int  gfc_device_code_version(int device, int *binary_version, int *ptx_version);
/* Self-check of the division the reference-arithmetic path uses where one divisor
 * serves several quotients (the explicit inverse's complex division, SU3_ops.c:843-900):
 * compares it bit for bit with IEEE division on `count` pseudo-random operand pairs
 * from `seed` and stores the number of differing quotients (0 expected).
 * Synchronous.  No counterpart in the reference. */
int  gfc_check_division(int device, unsigned long long seed, long long count, unsigned long long *mismatches);
/* page-locked host memory for fast transfers (cudaMallocHost / cudaFreeHost) */
void *gfc_host_alloc(size_t bytes);
void  gfc_host_free(void *p);
int  gfc_ctx_create(int ns, int nt, int device, int flags, gfc_ctx **out);
int  gfc_ctx_destroy(gfc_ctx *c);
long long gfc_ctx_kernel_launches(const gfc_ctx *c);
void *gfc_ctx_stream(gfc_ctx *c);   /* the context's cudaStream_t, as void* */
int  gfc_ctx_sync(gfc_ctx *c);   /* waits for all work and copies queued on the context */

/* Links in, as raw file bytes in the reference order: elem_bytes 8 (FP64) or 4
 * (FP32, converted to FP64 like CONV_CFG_TO_WORKING_PRECISION), byteswap 1 for
 * big-endian files (NEED_BYTE_SWAP_IN).  Pinned host memory is copied directly;
 * other memory goes through pinned staging.  Swap and conversion run on the GPU. */
int  gfc_ctx_upload_links(gfc_ctx *c, const void *host, int elem_bytes, int byteswap);
/* loadConfig + reunitarizeField (gauge_fix_coulomb.c:123-131) fused: the links as
 * gfc_ctx_upload_links then gfc_ctx_reunitarize give them, in one pass */
int  gfc_ctx_upload_links_reunit(gfc_ctx *c, const void *host, int elem_bytes, int byteswap);
int  gfc_ctx_download_links(gfc_ctx *c, void *host, int elem_bytes, int byteswap);
int  gfc_ctx_upload_gt(gfc_ctx *c, const void *host, int elem_bytes, int byteswap);
int  gfc_ctx_download_gt(gfc_ctx *c, void *host, int elem_bytes, int byteswap);
/* gfc_ctx_download_gt left in flight on the context's streams, so that a pipeline
 * can read one lattice's G while another context fixes the next: host must be
 * page-locked (gfc_host_alloc), else GFC_ERR_ARG; gfc_ctx_sync completes it, and
 * later calls on the context are ordered after it.  No counterpart in the reference
 * (writeGaugeTransf, fields_io.c:493-565, writes synchronously). */
int  gfc_ctx_download_gt_async(gfc_ctx *c, void *host, int elem_bytes, int byteswap);

/* one link (mu = 0 temporal, 1..3 z,y,x) at lexicographic site L, 18 doubles
 * (getLink, fields.c:233-271) */
int  gfc_ctx_get_link(gfc_ctx *c, size_t site, int mu, double *out18);

/* reunitarizeField (fields.c:144-187) on all 4V links */
int  gfc_ctx_reunitarize(gfc_ctx *c);
/* device-side copy of all links and its restore (restart a fix without a host transfer) */
int  gfc_ctx_save_links(gfc_ctx *c);
int  gfc_ctx_restore_links(gfc_ctx *c);
/* reunitarizeField(G, V) */
int  gfc_ctx_reunitarize_gt(gfc_ctx *c);
/* setFieldToIdentity (fields.c:64-100) on G */
int  gfc_ctx_set_identity_gt(gfc_ctx *c);
/* device status word (GFC_STATUS_* bits: 1 projection failure, 2 NaN), then cleared */
int  gfc_ctx_status(gfc_ctx *c, unsigned *status);

/* calculate_e2 / calculateTheta (gauge_fixing.c:341-442), calculateF (289-337),
 * averagePlaquette spatial / temporal (measurement.c:108-155) */
int  gfc_ctx_e2(gfc_ctx *c, double *e2, double *theta);
int  gfc_ctx_e2_slices(gfc_ctx *c, double *e2_per_slice);
int  gfc_ctx_functional(gfc_ctx *c, double *F);
int  gfc_ctx_plaquette(gfc_ctx *c, double *spatial, double *temporal);

/* n half-sweeps with indices first_sweep.. (parity = index & 1, as BLACKRED_SWEEP,
 * gauge_fixing.c:42), no reunitarisation, no stopping test; asynchronous */
int  gfc_ctx_halfsweeps(gfc_ctx *c, int first_sweep, int n, float omega_OR, unsigned hits, int precision);
/* apply G to the temporal links (U_t(x) <- G(x) U_t(x) G(x+t)^dagger) and reunitarise them */
int  gfc_ctx_finalize_temporal(gfc_ctx *c);
/* applyGaugeTransformationU (fields.c:375-435) with the resident G, on all links, in
 * the reference's arithmetic */
int  gfc_ctx_apply_gt(gfc_ctx *c);

/* ---- launch-shape autotuner (no counterpart in the reference) ------------------------ */
/* Times every compiled launch shape (threads per block x resident blocks per SM)
 * of the sweep kernels on this lattice and keeps the fastest for later fixes.
 * which: bit 0 exact FP64, bit 1 fast FP64, bit 2 FP32 (0 = all).  The links are
 * copied into the slot of gfc_ctx_save_links first (replacing any copy saved there
 * before) and restored from it after the timing, so the context's links are as
 * before and a later gfc_ctx_restore_links returns them; G is reset to the
 * identity.  times (may be NULL) receives seconds per half-sweep:
 * [0..4] exact shapes (2 plain, 3 with the links staged in shared memory), [5..22]
 * fast FP64 shapes (9 plain, then 9 with links staged in shared memory by cp.async),
 * [23..40] FP32 shapes (same order), [41..44] fast FP64 slice-blocked candidates,
 * [45..48] FP32 slice-blocked candidates.  Slice
 * blocking runs a group of timeslices for several half-sweeps while its links stay in
 * L2 (timeslices share no link during the sweeps); it is kept only where it measured
 * faster. */
#define GFC_TUNE_SLOTS 49
int  gfc_ctx_autotune(gfc_ctx *c, int which, double *times);
int  gfc_ctx_get_shapes(const gfc_ctx *c, int *exact, int *fast64, int *fast32);
/* -1 keeps the current choice */
int  gfc_ctx_set_shapes(gfc_ctx *c, int exact, int fast64, int fast32);
/* slice blocking for the fast FP64 (bit 1) and/or FP32 (bit 2) sweeps: groups of
 * `slices` timeslices, `sweeps` half-sweeps per visit (0 / 1: no blocking) */
int  gfc_ctx_set_blocking(gfc_ctx *c, int precision_bits, int slices, int sweeps);
int  gfc_ctx_get_blocking(const gfc_ctx *c, int *slices64, int *sweeps64, int *slices32, int *sweeps32);

/* ---- allocation-free observable --------------------------------------------------- */
/* e2 and theta (the quantities of gfc_ctx_e2) of links the caller already holds in
 * device memory on the current device, in the reference layout (4V*18 doubles),
 * without allocating any device memory: for callers that cannot let a library call
 * cudaMalloc/cudaFree (their allocator owns the GPU's memory, or a device-wide
 * synchronisation from cudaFree would stall other work sharing the GPU).  No
 * counterpart in the reference.  Scratch is a fixed 128 KiB array inside the
 * library (GFC_NOALLOC_SCRATCH_DOUBLES doubles per GPU, held until exit); lattices
 * whose partial sums do not fit are rejected with GFC_ERR_ARG and a message in
 * gfc_last_error().  Calls share that array: calls that overlap on the GPU race.
 * The first call on a device looks up the array's address (cudaGetSymbolAddress).
 * stream is a cudaStream_t (NULL: the legacy default stream).
 * The call is synchronous: it copies e2 and theta to the host and waits for them.
 * u_dev must be device memory of the current device or managed memory
 * (cudaPointerGetAttributes is asked first); host memory and another GPU's memory
 * are refused with GFC_ERR_ARG before any kernel runs. */
#define GFC_NOALLOC_SCRATCH_DOUBLES 16384
int  gfc_e2_theta_device_noalloc(int ns, int nt, const double *u_dev, void *stream, double *e2, double *theta);

/* ---- batches: many lattices, per-timeslice retirement (no counterpart in the reference) ---- */
/* A batch holds up to max_slots lattices (nt <= max_nt, max_sites sites in total) on
 * one GPU.  Every timeslice of every lattice is swept independently (timeslices
 * share no link during the sweeps) and retires when its own e2 falls below the
 * tolerance (measured on the links it keeps); with GFC_PREC_MIXED it first runs FP32
 * bulk sweeps until its e2 falls below options.switch_e2 and is then rebuilt in
 * FP64.  Lattices of odd ns run in FP64 whatever the precision asked for, each
 * half-sweep in four launches over the boundary levels that keep the reference's
 * sequential order where same-parity sites share a link.  One round = K
 * half-sweeps of all active timeslices, replayed as a captured CUDA graph.  Slots
 * can be added, activated, finalised and removed between rounds (continuous
 * batching).  Slot memory is allocated stream-ordered (no device synchronisation). */
typedef struct gfc_batch gfc_batch;
int    gfc_batch_create(int device, size_t max_sites, int max_slots, int max_nt, gfc_batch **out);
int    gfc_batch_destroy(gfc_batch *b);
size_t gfc_batch_slot_bytes(int ns, int nt);          /* device bytes one slot needs */
int    gfc_batch_add(gfc_batch *b, int ns, int nt, int *slot);   /* GFC_ERR_BUSY when full */
int    gfc_batch_remove(gfc_batch *b, int slot);
/* hold != 0: keep the slot resident but out of the rounds (its state is kept, so
 * holding changes when it finishes, not what it computes); 0: sweep it again */
int    gfc_batch_hold(gfc_batch *b, int slot, int hold);
/* links in (raw reference-layout bytes, as gfc_ctx_upload_links), reunitarised */
int    gfc_batch_upload(gfc_batch *b, int slot, const void *host, int elem_bytes, int byteswap);
/* the seeded synthetic configuration of gfc_synth_config built on the device
 * (same construction and streams; equal to the host one up to rounding), reunitarised */
int    gfc_batch_synth(gfc_batch *b, int slot, uint64_t seed, double scale);
/* G = 1; start fixing this slot from the next round (GFC_PREC_MIXED: FP32 first) */
int    gfc_batch_activate(gfc_batch *b, int slot, int precision);
/* one round; *active = timeslices still working */
int    gfc_batch_round(gfc_batch *b, const gfc_params *p, const gfc_options *o, int *active);
int    gfc_batch_slot_done(gfc_batch *b, int slot, int *done);
/* retired slot: canonical FP64 links and G, reunitarised, temporal links transformed;
 * report: sweeps = largest per-timeslice half-sweep count, e2, theta, functional */
int    gfc_batch_finalize(gfc_batch *b, int slot, gfc_report *r);
int    gfc_batch_plaquette(gfc_batch *b, int slot, double *spatial, double *temporal);
int    gfc_batch_download_gt(gfc_batch *b, int slot, void *host, int elem_bytes, int byteswap);
int    gfc_batch_download_links(gfc_batch *b, int slot, void *host, int elem_bytes, int byteswap);
int    gfc_batch_status(gfc_batch *b, unsigned *status);
/* half-sweeps each timeslice of the slot has received (nt ints) */
int    gfc_batch_slice_sweeps(gfc_batch *b, int slot, int *out);
long long gfc_batch_kernel_launches(const gfc_batch *b);
void  *gfc_batch_stream(gfc_batch *b);
/* minimum resident CTAs per SM of the FP32 / FP64 sweep kernels and half-sweeps per
 * round: 1..4 CTAs of 128 threads, or 8, 11 or 12 one-warp CTAs (links staged in
 * shared memory, the 128 sites of a work item swept 32 at a time) */
int    gfc_batch_set_shape(gfc_batch *b, int minb32, int minb64, int round_sweeps);
/* FP64 batch sweep with the links staged in shared memory (1, default) or not (0) */
int    gfc_batch_set_staging(gfc_batch *b, int stage64);
int    gfc_batch_get_shape(const gfc_batch *b, int *minb32, int *minb64, int *stage64, int *round_sweeps);
/* Time the launch shapes on a scratch lattice of size ns^3 x nt and keep the fastest
 * (FP32 resident CTAs per SM, FP64 resident CTAs and staging, half-sweeps per round).
 * Needs a batch without activated slots.  times (may be NULL): seconds per half-sweep,
 * [0..2] FP32 minb 2,3,4; [3..7] FP64 (minb, staged) (2,0) (3,0) (4,0) (2,1) (3,1);
 * [8..10] rounds of 4, 8, 16 half-sweeps; [11..13] FP32 one-warp CTAs 8, 11, 12 per
 * SM; [14..16] FP64 one-warp CTAs 8, 11, 12 per SM. */
#define GFC_BATCH_TUNE_SLOTS 17
int    gfc_batch_autotune(gfc_batch *b, int ns, int nt, double *times);
/* rounds until every activated slot retired (or max_sweeps), then finalise them;
 * reports indexed by slot; returns the number of rounds */
int    gfc_batch_fix_all(gfc_batch *b, const gfc_params *p, const gfc_options *o, gfc_report *reports);

/* ---- serving: a request loop with continuous batching (no counterpart in the reference) ---- */
/* Requests queue on the host; gfc_server_step releases the device memory of
 * requests whose G has reached the host, admits queued requests in arrival order
 * with first fit while a slot and device memory are free, runs one batch round and
 * finalises requests whose timeslices have all retired.  A result thread copies
 * each finished G to host memory on its own stream while the next rounds run.
 * Requests join and leave while others are on the GPU; a request's result does
 * not depend on the others.  The gfc_server_* calls are made from one thread. */
typedef struct gfc_server gfc_server;
/* max_sites 0: capacity from mem_fraction of the free device memory */
int    gfc_server_create(int device, size_t max_sites, double mem_fraction, int max_slots, int max_nt,
                         gfc_server **out);
int    gfc_server_destroy(gfc_server *s);
size_t gfc_server_capacity_sites(const gfc_server *s);
/* links NULL: the seeded synthetic configuration, built on the device at admission */
int    gfc_server_submit(gfc_server *s, int ns, int nt, const void *links, int elem_bytes, int byteswap,
                         uint64_t seed, double scale, int precision, int64_t *id);
int    gfc_server_step(gfc_server *s, const gfc_params *p, const gfc_options *o, int *running, int *queued);
/* state 0 queued, 1 running (or G on its way to the host), 2 done (G on the host),
 * 3 fetched; times are seconds after submit */
int    gfc_server_poll(gfc_server *s, int64_t id, int *state, double *t_admit, double *t_done, gfc_report *report);
/* G of a done request (reference layout, FP64) in place: valid until released */
int    gfc_server_result(gfc_server *s, int64_t id, const double **gt, size_t *count);
/* copy G (elem_bytes 8 or 4; gt may be NULL) and, with release != 0, drop the host copy */
int    gfc_server_fetch(gfc_server *s, int64_t id, void *gt, int elem_bytes, int release);
/* pin `count` host buffers of `buffer_bytes` for results ahead of time (results
 * go to reused page-locked buffers, up to 32 GiB of them) */
int    gfc_server_reserve_host(gfc_server *s, size_t buffer_bytes, int count);
/* Scheduling of admitted requests (admission itself is by free memory either way):
 * GFC_SERVE_ALL (default) sweeps every admitted request in every round;
 * GFC_SERVE_SMALLEST_FIRST sweeps the requests still running smallest first, as many
 * as fit in work_sites sites (at least one), the others wait resident. */
#define GFC_SERVE_ALL            0
#define GFC_SERVE_SMALLEST_FIRST 1
int    gfc_server_set_policy(gfc_server *s, int policy, size_t work_sites);
/* host seconds in the phases of gfc_server_step (release, admission, rounds,
 * finalisation) and the rounds run */
int    gfc_server_stats(const gfc_server *s, double *seconds4, long long *rounds);
gfc_batch *gfc_server_batch(gfc_server *s);

/* gaugefixOverrelaxation (gauge_fixing.c:713-826) on the resident lattice:
 * sets G = 1, fixes U in place (spatial and temporal links), returns the number of
 * half-sweeps, GFC_FIX_NOT_CONVERGED (-1) or GFC_FIX_BAD_PARAMS (-2); a value below
 * -2 is a library error (gfc_last_error()).  opt may be NULL (reference behaviour). */
int  gfc_ctx_fix(gfc_ctx *c, const gfc_params *p, const gfc_options *opt, gfc_report *rep);

/* gaugefixOverrelaxation(U, G, params) (gauge_fixing.c:713-826, declared
 * gauge_fixing.h:67-69) on host arrays in the reference layout: U (4V matrices of
 * 9 complex doubles, native endian) is fixed in place and G (V matrices) receives
 * the transformation; a device context lives for the call.  Same return values as
 * gfc_ctx_fix; on -1 U and G are still written.  opt and rep may be NULL. */
int  gfc_gaugefix_overrelaxation(int ns, int nt, double *U, double *G, const gfc_params *p,
                                 const gfc_options *opt, gfc_report *rep, int device);

#ifdef __cplusplus
}
#endif
#endif /* GFC_H */
