/*
 * oracle_driver.h -- per-type-map driver of the CPU oracle (TEST INFRASTRUCTURE).
 * Starting line (main.f90:196-248) and the parallel level loop (the
 * reference runs its ATMOSPHERIC_LEVELS_LOOP serially, main.f90:81-180; levels
 * are independent, so the oracle may spread them over threads).
 */
#include <pthread.h>

static int SFX(starting_line)(const oracle_args *a, int64_t *idx, double *wv) {
  const unsigned char *recs = (const unsigned char *)a->records;
  double cut = (double)(real)a->cutoff;
  double v;
  int64_t i = 1;
  memcpy(&v, recs, 8);
  if (a->start_wv > cut) {
    double ext_start = a->start_wv - cut;
    while (v <= ext_start) {
      ++i;
      if (i > a->n_lines) return 9;
      memcpy(&v, recs + (size_t)(i - 1) * 36, 8);
    }
  }
  *idx = i;
  *wv = v;
  return 0;
}

typedef struct {
  const oracle_args *a;
  float *out;
  double *out64;
  int64_t *evals;
  int64_t idx;
  double wv;
  int next_level, status;
  pthread_mutex_t mu;
} SFX(pool_t);

/* Worker: takes the next unprocessed level until none is left. */
static void *SFX(level_worker)(void *arg) {
  SFX(pool_t) *p = (SFX(pool_t) *)arg;
  for (;;) {
    int lev, r;
    int64_t ev = 0;
    pthread_mutex_lock(&p->mu);
    lev = p->next_level++;
    pthread_mutex_unlock(&p->mu);
    if (lev >= p->a->n_levels) break;
    r = SFX(run_level)(p->a, lev, p->idx, p->wv, p->out, p->out64, &ev, -1, NULL);
    if (p->evals) p->evals[lev] = ev;
    if (r) {
      pthread_mutex_lock(&p->mu);
      if (!p->status) p->status = r;
      pthread_mutex_unlock(&p->mu);
    }
  }
  return NULL;
}

int SFX(oracle_run_map)(const oracle_args *a, float *out, double *out64, int64_t *evals) {
  SFX(pool_t) p;
  pthread_t th[256];
  int rc, n, i, started = 0;
  memset(&p, 0, sizeof p);
  rc = SFX(starting_line)(a, &p.idx, &p.wv);
  if (rc) return rc;
  p.a = a;
  p.out = out;
  p.out64 = out64;
  p.evals = evals;
  pthread_mutex_init(&p.mu, NULL);
  n = a->nthreads < 1 ? 1 : (a->nthreads > 256 ? 256 : a->nthreads);
  if (n > a->n_levels) n = a->n_levels;
  for (i = 1; i < n; ++i)
    if (pthread_create(&th[started], NULL, SFX(level_worker), &p) == 0) ++started;
  SFX(level_worker)(&p);
  for (i = 0; i < started; ++i) pthread_join(th[i], NULL);
  pthread_mutex_destroy(&p.mu);
  return p.status;
}

int SFX(oracle_dump_map)(const oracle_args *a, int level, int isub, double *dump) {
  int64_t idx;
  double wv;
  int rc = SFX(starting_line)(a, &idx, &wv);
  if (rc) return rc;
  return SFX(run_level)(a, level, idx, wv, NULL, NULL, NULL, isub, dump);
}

int SFX(oracle_shape_map)(const oracle_args *a, int level, int64_t line, double X, double *v,
                          int *region) {
  return SFX(shape_probe)(a, level, line, X, v, region);
}

int SFX(oracle_windows_map)(const oracle_args *a, int64_t *lo, int64_t *hi) {
  const unsigned char *recs = (const unsigned char *)a->records;
  int64_t idx, line_idx;
  double wv, s = a->start_wv, cut = (double)(real)a->cutoff;
  int rc = SFX(starting_line)(a, &idx, &wv), isub = 0;
  if (rc) return rc;
  line_idx = idx;
  while (s < a->end_wv) {
    double ext_end = s + DELTA_WV + cut, cap = (s - cut) + DELTA_WV, v;
    int64_t I;
    if (cap <= wv) cap = wv;
    lo[isub] = line_idx;
    for (I = line_idx;; ++I) {
      if (I > a->n_lines) return 9;
      memcpy(&v, recs + (size_t)(I - 1) * 36, 8);
      if (v >= ext_end) break;
      if (v <= cap) line_idx = I;
    }
    hi[isub] = I;
    s = s + DELTA_WV;
    ++isub;
  }
  return 0;
}
