/*
 * marfa_gpu.h -- C ABI of the B200 line-by-line library (libmarfa_gpu.so).
 *
 * This is the drop-in boundary for MARFA's line-by-line core.  In the
 * reference the core is driven from app/main.f90 through module globals:
 *   - readCommandLineArguments / readAtmosphericParameters / readTIPS set the
 *     run (EnvironmentSetup.f90:34-95, :169-184; Atmsosphere.f90:29-60);
 *   - for every level and 10 cm-1 subinterval, main.f90:148-168 calls
 *     resetAbsorptionGridValues, lblScheme(lineIdx, capWV) (LBL.f90:25),
 *     cascadeInterpolation (Grids.f90:104) and writes one PT record;
 *   - the line shape and the chi-factor are plugged in through the abstract
 *     interfaces `shape(nu)` and `chifactor(nu, moleculeIntCode)`
 *     (Interfaces.f90:5-23) selected by setShapeFunction / setChiFactorFunction
 *     (Shapes.f90:11-15; ChiFactors.f90:11-16).
 * Here one call computes every record of every level; shapes and chi-factors
 * are selected by enum.  All pointers are plain host pointers unless a name
 * says `device`; no pointer is kept after a call returns.  Every function
 * returns a status: 0 on success, the reference's `stop` code for the same
 * failure (6: more than 200 levels, 8: unsupported molecule, 9: line database
 * ended inside a window), or one of the MARFA_E* codes below.  One context
 * per host thread; calls on one context are serialised on its stream.
 */
#ifndef MARFA_GPU_H
#define MARFA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes beyond the reference's stop codes 1..9 */
#define MARFA_OK 0
#define MARFA_E_DB 9            /* line list ended before a window closed (LBL.f90:41-57) */
#define MARFA_E_ARG 10          /* invalid argument                                  */
#define MARFA_E_TEMPERATURE 11  /* level temperature outside the TIPS table          */
#define MARFA_E_UNSORTED 12     /* line list not sorted by wavenumber                */
#define MARFA_E_ISOTOPE 13      /* jointMolIso/100 outside the WISO/TIPS tables      */
#define MARFA_E_CAPACITY 15     /* input beyond a fixed capacity: the storage of     */
                                /* marfa_compute_record_static, or more than 65535   */
                                /* lines within 1 cm-1 of one subinterval            */
#define MARFA_E_CUDA 100        /* CUDA runtime error (see marfa_last_error)         */
#define MARFA_E_NOMEM 101       /* device allocation failed                          */
#define MARFA_E_NODEVICE 110    /* no CUDA device                                    */

/* line shapes (Shapes.f90:8-15): VOIGT is `voigt` (Shapes.f90:22-133),
 * LORENTZ is `lorentzShape` (Shapes.f90:135-141), the chi-corrected Lorentz
 * at every offset.  ONE and ABSX are diagnostic shapes (F = 1 and F = |X|)
 * used to check the multigrid placement exactly. */
#define MARFA_SHAPE_VOIGT 0
#define MARFA_SHAPE_LORENTZ 1
#define MARFA_SHAPE_ONE 100
#define MARFA_SHAPE_ABSX 101

/* chi-factors (ChiFactors.f90:18-122); applied only when mol_code == 2 */
#define MARFA_CHI_NONE 0
#define MARFA_CHI_TONKOV 1
#define MARFA_CHI_POLLACK 2
#define MARFA_CHI_PERRIN 3

/* target value (EnvironmentSetup.f90:60-94): ACS writes RK, VAC density*RK */
#define MARFA_TARGET_ACS 0
#define MARFA_TARGET_VAC 1

/* arithmetic of the line-shape accumulation */
#define MARFA_PREC_FP64 0   /* every quantity in double: the drop-in          */
#define MARFA_PREC_FP32C 1  /* FP32 shapes and FP32 partial sums reduced in   */
                            /* double; FP64 prep, offsets and cascade         */

#define MARFA_NT 20481      /* points per PT record (Grids.f90:16)            */

typedef struct marfa_ctx marfa_ctx;

/* One 36-byte little-endian line record, as in the reference's databases
 * (LBL.f90:43-44; processParFile.f90:140-176). */
#pragma pack(push, 1)
typedef struct {
  double nu;        /* transition wavenumber [cm-1]                 */
  float S;          /* intensity at 296 K                           */
  float gamma_air;  /* foreign-broadened HWHM at 296 K [cm-1/atm]   */
  float gamma_self; /* self-broadened HWHM [cm-1/atm]               */
  float e_lower;    /* lower-state energy [cm-1]                    */
  float n_air;      /* temperature exponent of gamma_air            */
  int32_t joint_mol_iso; /* isotopologue index * 100 + molecule     */
  float delta_air;  /* pressure shift [cm-1/atm]                    */
} marfa_line_record;
#pragma pack(pop)

/* Run parameters: the 7 positional arguments of `marfa` (README.md:195-207)
 * plus the options the reference fixes at compile time. */
typedef struct {
  double start_wv, end_wv; /* Vstart, Vend [cm-1]                              */
  double cutoff;           /* CutOff [cm-1]                                    */
  int target;              /* MARFA_TARGET_*                                   */
  int mol_code;            /* getSpeciesCode of the molecule (2 = CO2)         */
  int chi;                 /* MARFA_CHI_*                                      */
  int shape;               /* MARFA_SHAPE_*                                    */
  int precision;           /* MARFA_PREC_*                                     */
} marfa_run;

/* Create a context on `device`: uploads the line list (sorted by nu; the last
 * record should be a sentinel beyond every window), the TIPS table
 * ([n_iso][n_temp], T = 20 + 2j K; reference layout of TIPS(74, 501)) and
 * sizes the device buffers.  Replaces readTIPS (EnvironmentSetup.f90:169-184)
 * and the database open of determineStartingSpectralLine (main.f90:196-212). */
int marfa_ctx_create(const marfa_line_record *lines, int64_t n_lines, const double *tips,
                     int n_iso, int n_temp, int device, marfa_ctx **out);
void marfa_ctx_destroy(marfa_ctx *ctx);
const char *marfa_last_error(const marfa_ctx *ctx);

/* Temperature grid of the context's TIPS table: node j (0-based) at
 * t_first + j * t_step K.  The default, 20 K and 2 K, is the grid of the
 * reference's table (TIPS(74, 501), Gamache 2017; Spectroscopy.f90:91-115).
 * The reference plans Gamache's 2021 partition sums (README.md:458-460),
 * which come on 1 K steps: pass such a table as `tips` to marfa_ctx_create
 * (isotopologues as rows, NaN beyond an isotopologue's last temperature) and
 * set its grid here.  Q(T) is interpolated linearly between the nodes around
 * T, as the reference does on its grid, and Q(296 K) is the node at 296 K
 * when there is one.  296 K must lie inside the table (else MARFA_E_ARG);
 * a level temperature outside it returns MARFA_E_TEMPERATURE.  Graphs
 * captured before the change are refused afterwards (status 10). */
int marfa_ctx_set_tips_grid(marfa_ctx *ctx, double t_first, double t_step);

/* Number of subintervals of [start_wv, end_wv) (main.f90:117-122) and the
 * PT record number of subinterval `isub` (main.f90:126). */
int marfa_num_subintervals(double start_wv, double end_wv);
int marfa_record_number(double start_wv, int isub);

/* Line window of every subinterval without a device: lo[isub], hi[isub]
 * (0-based, hi exclusive) are the first line read and the line that ends the
 * scan in lblScheme (LBL.f90:41-61, capWV of main.f90:138-144, starting
 * line of main.f90:196-248).  nu: the sorted line centres.  Returns 9 when
 * the list ends inside a window. */
int marfa_plan_windows(const double *nu, int64_t n_lines, double start_wv, double end_wv,
                       double cutoff, int64_t *lo, int64_t *hi);

/* All levels x all subintervals of one profile: replaces the
 * ATMOSPHERIC_LEVELS_LOOP / SUBINTERVALS_LOOP of main.f90:81-180.
 * pressure [atm], temperature [K], density [1/(cm^2 km)] per level (<= 200).
 * out: host [n_levels][n_sub][MARFA_NT] float32 records;
 * out64 (optional): the same before the final rounding to float32. */
int marfa_compute(marfa_ctx *ctx, const marfa_run *run, const double *pressure,
                  const double *temperature, const double *density, int n_levels,
                  float *out, double *out64);

/* Many profiles with uneven level counts in one batched launch sequence.
 * level_counts[n_profiles]; pressure/temperature/density are concatenated
 * over profiles; out is [sum(level_counts)][n_sub][MARFA_NT]. */
int marfa_compute_batched(marfa_ctx *ctx, const marfa_run *run, int n_profiles,
                          const int *level_counts, const double *pressure,
                          const double *temperature, const double *density, float *out,
                          double *out64);

/* Same as marfa_compute_batched with a DEVICE output buffer, enqueued on
 * `stream` (a cudaStream_t; NULL = the context's stream) and returning
 * without waiting; the inputs are host arrays copied inside the call (through
 * a ring of four pinned buffers: up to four calls queue ahead of the device
 * before a call waits).  Consecutive calls on one context use one stream: the
 * per-call tables live in the context. */
int marfa_compute_device(marfa_ctx *ctx, const marfa_run *run, int n_profiles,
                         const int *level_counts, const double *pressure,
                         const double *temperature, const double *density,
                         float *device_out, void *stream);
int marfa_synchronize(marfa_ctx *ctx);

/* A compute call captured once into a CUDA graph and replayed for new
 * profiles of the same shape.  The reference recomputes from scratch for
 * every profile (main.f90:81-180); this is the batched form for many
 * profiles.  marfa_graph_create computes the records of the given profiles
 * into `device_out` (like marfa_compute_device, then waits), then captures the
 * same launches -- prep, sort, far, persistent fine kernel with its device
 * work queue, cascade -- into a graph.  marfa_graph_launch takes new
 * pressure / temperature / density arrays of the same level counts, stages
 * them and launches the graph on `stream` (NULL = the context's stream)
 * without waiting; the records go to the same `device_out`.  It returns
 * MARFA_E_ARG when the launch plan no longer matches the capture (the
 * context's buffers were grown by a larger computation in between, or the
 * near-line counts of the new profile need larger staging): create a new
 * graph then.  One graph per context at a time is launched on its stream. */
typedef struct marfa_graph marfa_graph;
int marfa_graph_create(marfa_ctx *ctx, const marfa_run *run, int n_profiles,
                       const int *level_counts, const double *pressure,
                       const double *temperature, const double *density, float *device_out,
                       marfa_graph **out);
int marfa_graph_launch(marfa_graph *graph, const double *pressure, const double *temperature,
                       const double *density, void *stream);
void marfa_graph_destroy(marfa_graph *graph);

/* Chooses the context's launch parameters that do not change the method --
 * lines per far-kernel block (far_chunk: 2048, 4096, 8192 or 16384) and the number of
 * coarse fine grids whose accumulators are summed by groups of lanes rather
 * than one thread each (coop_k: 1..5) -- by timing every candidate on up to sixteen levels of the given
 * profile; for FP32c it then times the other fine-kernel block shape
 * (fine_pair, see marfa_ctx_set_launch) at the best of those.  Keeps the
 * fastest in the context and returns far_chunk and coop_k (the shape through
 * marfa_ctx_get_launch).  Results change only by summation order (far-line
 * sums are split differently).  No reference counterpart (the reference has
 * no launch parameters). */
int marfa_autotune(marfa_ctx *ctx, const marfa_run *run, int n_levels, const double *pressure,
                   const double *temperature, const double *density, int *far_chunk,
                   int *coop_k);

/* Sets the context's launch parameters (as chosen by marfa_autotune, for
 * example to reuse a tuning across processes): far_chunk (2048, 4096, 8192 or
 * 16384), coop_k (1..5) and fine_pair (0: FP32c units with many near lines
 * run on one 1024-thread fine block per SM; 1: on two 512-thread blocks per
 * SM; FP64 ignores it).  Returns MARFA_E_ARG for any other value.  Graphs
 * captured before the change keep their launch plan and are refused on
 * replay when it differs. */
int marfa_ctx_set_launch(marfa_ctx *ctx, int far_chunk, int coop_k, int fine_pair);
/* The context's current launch parameters (any pointer may be NULL). */
int marfa_ctx_get_launch(marfa_ctx *ctx, int *far_chunk, int *coop_k, int *fine_pair);

/* Replaces the reference intensities S and air-broadening coefficients
 * gamma_air of every line by double values (either pointer may be NULL: back
 * to the database record's float value).  The reference reads both from the
 * line record (LBL.f90:43-44); this is the parameter update of a retrieval
 * that differentiates with respect to them (marfa_vjp). */
int marfa_ctx_set_line_params(marfa_ctx *ctx, const double *S, const double *gamma_air);

/* Vector-Jacobian product of the records.  For the cotangent
 * cotangent[n_levels][n_sub][MARFA_NT] (host, double) of the FP64 records
 * (out64 of marfa_compute) it returns dL/dT and dL/dP per level and dL/dS and
 * dL/dgamma_air per line (host arrays [n_levels] and [n_lines]) of
 * L = sum cotangent * record, holding the placement of each line, the
 * Humlicek region choices and the cascade clamp decisions fixed.  The line
 * shape is recomputed, nothing of the forward pass is stored.  Voigt shape
 * only; run->precision is ignored (FP64).  No reference counterpart: the
 * reference has no derivatives. */
int marfa_vjp(marfa_ctx *ctx, const marfa_run *run, const double *pressure,
              const double *temperature, const double *density, int n_levels,
              const double *cotangent, double *d_temperature, double *d_pressure,
              double *d_S, double *d_gamma_air);

/* Number of line-shape evaluations the reference schedule performs for this
 * workload (FSHAPE calls of LineGridCalc.f90), per level; far_per_level
 * (optional) receives the part made by lines at least 1 cm-1 outside their
 * subinterval (21 grid-0 evaluations each). */
int marfa_eval_count(marfa_ctx *ctx, const marfa_run *run, int n_levels,
                     const double *pressure, const double *temperature, const double *density,
                     int64_t *evals_per_level, int64_t *far_per_level);

/* Raw accumulators of one (level, subinterval) after the line loop and
 * before the cascade: [MARFA_NT] RK, then P, M, L of grids 0..9 (10230 cells
 * each, grid k at offset 10*(2^k-1)); doubles. */
int marfa_debug_accumulators(marfa_ctx *ctx, const marfa_run *run, const double *pressure,
                             const double *temperature, const double *density, int n_levels,
                             int level, int isub, double *dump);

/* Timing of the last compute call, measured with CUDA events on the stream
 * it ran on (waits for that call to finish): times[8] = milliseconds of each
 * kernel family (prep, sort, far, fine, cascade), the total, the number of
 * kernel launches and the number of far-kernel launches. */
int marfa_last_timings(marfa_ctx *ctx, double *times);

/* One PT record (one level, one subinterval) computed without allocating any
 * memory.  This entry point has no counterpart in the reference, which
 * computes whole profiles; it exists for callers that cannot call cudaMalloc,
 * for example applications whose device memory is owned by a pool allocator
 * that reserves the GPU at start-up, or loops that cannot afford
 * cudaMalloc's implicit device synchronisation.  All device working storage
 * is one static array of MARFA_STATIC_SCRATCH_BYTES inside the library, held
 * by every GPU that loads the library until the process exits.
 *   lines, n_lines: all line records, sorted by centre (as the reference's
 *   databases are) and ending beyond the last window; the window of
 *   subinterval `isub` is found by binary searches, and only its records are
 *   checked for order (MARFA_E_UNSORTED) and copied to the device (at most
 *   MARFA_STATIC_MAX_WINDOW_LINES lines, of which at most
 *   MARFA_STATIC_MAX_NEAR_LINES within 1 cm-1 of the subinterval when they do
 *   not fit on chip) is copied to the device; larger inputs return
 *   MARFA_E_CAPACITY.
 *   tips: [n_iso][n_temp] (at most 131,072 values); pressure, temperature,
 *   density: the level; record: 20481 floats, host or device memory.
 *   stream: cudaStream_t or NULL; the call waits for its work to finish
 *   (it synchronises the stream and copies from pageable host memory, so it
 *   cannot be called on a stream that is being captured into a graph).
 *   msg (optional): receives a text description of a failure.
 * Every call looks up the array's device address on the current device (the
 * first call on a device also loads the library's device code there).  Every
 * call on a device reuses the same array: calls that overlap on the GPU
 * (from two host threads, or on two streams) race, so callers serialise
 * them. */
#define MARFA_STATIC_MAX_WINDOW_LINES 65536
#define MARFA_STATIC_MAX_NEAR_LINES 8192
#define MARFA_STATIC_SCRATCH_BYTES (12u * 1024u * 1024u)
int marfa_compute_record_static(const marfa_line_record *lines, int64_t n_lines, const double *tips,
                                int n_iso, int n_temp, const marfa_run *run, double pressure,
                                double temperature, double density, int isub, float *record,
                                void *stream, char *msg, size_t msg_len);

#ifdef __cplusplus
}
#endif
#endif
