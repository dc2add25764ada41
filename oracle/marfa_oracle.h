/*
 * marfa_oracle.h -- CPU ORACLE for the MARFA line-by-line core.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * Fortran algorithm (Razumovskyy/MARFA, src/ and app/main.f90) used as the
 * checker for the CUDA library and as the timed CPU baseline.  Nothing in the
 * product path links, loads or calls it; only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg do.
 *
 * Parity pin: the reference ships no golden PT-tables and no Voigt known-answer
 * tests (its test/ folder only holds the .par -> 36-byte record pair), and no
 * Fortran compiler exists in this image, so the restatement cannot be checked
 * against reference outputs.  PARITY UNPINNED against the Fortran build; it is
 * pinned instead against (a) the reference's 36-byte record fixture
 * (test/testDB.02), (b) region-by-region formula checks and a loose
 * scipy.special.wofz accuracy bound, (c) eval-count and brute-force properties
 * of the multigrid, all in tests/.
 *
 * Two type maps are built from one source (oracle_impl.h):
 *   mixed : Fortran `real` -> float, `real(kind=DP)` -> double, with Fortran's
 *           promotion rules and operation order (the reference as shipped);
 *   fp64  : every quantity and constant in double (the FP64 reference used for
 *           error statistics).
 */
#ifndef MARFA_ORACLE_H
#define MARFA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_MIXED = 0, ORACLE_FP64 = 1 };
enum { ORACLE_CHI_NONE = 0, ORACLE_CHI_TONKOV = 1, ORACLE_CHI_POLLACK = 2, ORACLE_CHI_PERRIN = 3 };
enum { ORACLE_SHAPE_VOIGT = 0, ORACLE_SHAPE_LORENTZ = 1, ORACLE_SHAPE_ONE = 100, ORACLE_SHAPE_ABSX = 101 };
enum { ORACLE_TARGET_ACS = 0, ORACLE_TARGET_VAC = 1 };

/* Layout of one (level, subinterval) accumulator dump (doubles):
 *   [0, 20481)            RK(1..NT)        finest grid, direct contributions
 *   [20481, +10230)       P  of grids 0..9 (grid k at offset 10*(2^k-1))
 *   [.., +10230)          M  (RK0, RK1 ... in the reference)
 *   [.., +10230)          L                                                  */
#define ORACLE_NT 20481
#define ORACLE_NCELLS 10230
#define ORACLE_DUMP_LEN (ORACLE_NT + 3 * ORACLE_NCELLS)

typedef struct {
  const void *records;     /* n_lines 36-byte little-endian line records        */
  int64_t n_lines;
  const double *tips;      /* [n_iso][n_temp] partition sums, T = t0 + dt*j    */
  int n_iso, n_temp;
  double tips_t0, tips_dt; /* the table's grid (the reference's: 20 K, 2 K)    */
  const double *pressure;  /* [n_levels] atm                                   */
  const double *temperature;/* [n_levels] K                                    */
  const double *density;   /* [n_levels] molecules / (cm^2 km)                 */
  int n_levels;
  double start_wv, end_wv; /* cm-1                                              */
  double cutoff;           /* cm-1 (Fortran `real`; rounded to float in mixed) */
  int target;              /* ORACLE_TARGET_*                                  */
  int chi;                 /* ORACLE_CHI_*                                     */
  int mol_code;            /* getSpeciesCode integer (2 = CO2)                  */
  int shape;               /* ORACLE_SHAPE_*                                   */
  int precision;           /* ORACLE_MIXED / ORACLE_FP64                       */
  int nthreads;            /* levels run in parallel over this many threads   */
} oracle_args;

/* Number of 10 cm-1 subintervals of [start_wv, end_wv) (main.f90:122). */
int oracle_num_subintervals(double start_wv, double end_wv);
/* PT record number of subinterval `isub` (main.f90:126). */
int oracle_record_number(double start_wv, int isub);

/* Full run.  out: [n_levels][n_sub][NT] float32 records as written to the
 * .ptbin files; out64 (optional): the same values before the final rounding
 * to float32 (fp64 map) or widened floats (mixed map).  evals (optional):
 * [n_levels] number of line-shape calls in the reference schedule.  Returns 0
 * or a reference-style status code (9: line list ended inside a window;
 * 10: bad argument; 11: temperature outside the TIPS table; 12: lines not
 * sorted; 13: isotopologue outside the tables). */
int oracle_run(const oracle_args *a, float *out, double *out64, int64_t *evals);

/* Raw accumulators of one (level, subinterval) after the line loop and before
 * the cascade, in the ORACLE_DUMP_LEN layout above. */
int oracle_unit_accumulators(const oracle_args *a, int level, int isub, double *dump);

/* Per-line shape-function value F(X) for one line at one level (diagnostics
 * and region tests); region (optional) receives 0..4 or 40/41/42 for the three
 * region-4 branches. */
int oracle_shape_value(const oracle_args *a, int level, int64_t line, double X,
                       double *value, int *region);

/* Line window [first, last] (1-based, inclusive of the exit record) of each
 * subinterval: lo[isub] = first record read, hi[isub] = record that ended the
 * scan (its nu >= extEnd). */
int oracle_windows(const oracle_args *a, int64_t *lo, int64_t *hi);

#ifdef __cplusplus
}
#endif
#endif
