/* oracle_api.c -- public entry points of the CPU oracle (TEST INFRASTRUCTURE). */
#include <math.h>
#include <string.h>
#include "marfa_oracle.h"

int oracle_run_map_mixed(const oracle_args *, float *, double *, int64_t *);
int oracle_run_map_fp64(const oracle_args *, float *, double *, int64_t *);
int oracle_dump_map_mixed(const oracle_args *, int, int, double *);
int oracle_dump_map_fp64(const oracle_args *, int, int, double *);
int oracle_shape_map_mixed(const oracle_args *, int, int64_t, double, double *, int *);
int oracle_shape_map_fp64(const oracle_args *, int, int64_t, double, double *, int *);
int oracle_windows_map_mixed(const oracle_args *, int64_t *, int64_t *);
int oracle_windows_map_fp64(const oracle_args *, int64_t *, int64_t *);

/* SUBINTERVALS_LOOP, main.f90:117-122, 171-172 */
int oracle_num_subintervals(double start_wv, double end_wv) {
  int n = 0;
  double s = start_wv;
  while (s < end_wv) {
    ++n;
    s = s + 10.0;
  }
  return n;
}

/* outputRecNum = (startDeltaWV + 1.0) / 10.0, main.f90:126 */
int oracle_record_number(double start_wv, int isub) {
  double s = start_wv;
  int i;
  for (i = 0; i < isub; ++i) s = s + 10.0;
  return (int)((s + 1.0) / 10.0);
}

static int check(const oracle_args *a) {
  const unsigned char *r = (const unsigned char *)a->records;
  int64_t i;
  double prev, v;
  if (!a || !a->records || a->n_lines < 1 || !a->tips || a->n_levels < 0) return 10;
  if (a->n_temp < 139 || a->n_iso < 1) return 10;
  memcpy(&prev, r, 8);
  for (i = 1; i < a->n_lines; ++i) {
    memcpy(&v, r + (size_t)i * 36, 8);
    if (v < prev) return 12;
    prev = v;
  }
  return 0;
}

int oracle_run(const oracle_args *a, float *out, double *out64, int64_t *evals) {
  int rc = check(a);
  if (rc) return rc;
  return a->precision == ORACLE_FP64 ? oracle_run_map_fp64(a, out, out64, evals)
                                     : oracle_run_map_mixed(a, out, out64, evals);
}

int oracle_unit_accumulators(const oracle_args *a, int level, int isub, double *dump) {
  int rc = check(a);
  if (rc) return rc;
  if (level < 0 || level >= a->n_levels || isub < 0 ||
      isub >= oracle_num_subintervals(a->start_wv, a->end_wv))
    return 10;
  return a->precision == ORACLE_FP64 ? oracle_dump_map_fp64(a, level, isub, dump)
                                     : oracle_dump_map_mixed(a, level, isub, dump);
}

int oracle_shape_value(const oracle_args *a, int level, int64_t line, double X, double *value,
                       int *region) {
  if (!a || line < 0 || line >= a->n_lines || level < 0 || level >= a->n_levels) return 10;
  return a->precision == ORACLE_FP64 ? oracle_shape_map_fp64(a, level, line, X, value, region)
                                     : oracle_shape_map_mixed(a, level, line, X, value, region);
}

int oracle_windows(const oracle_args *a, int64_t *lo, int64_t *hi) {
  int rc = check(a);
  if (rc) return rc;
  return a->precision == ORACLE_FP64 ? oracle_windows_map_fp64(a, lo, hi)
                                     : oracle_windows_map_mixed(a, lo, hi);
}
