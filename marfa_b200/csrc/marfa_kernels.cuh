// marfa_kernels.cuh -- launch interface between the host driver and the kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "marfa_device.cuh"

namespace marfa {

// SoA copy of the line list (line-index order, index 0 = record 1).
struct DeviceLines {
  const double *nu;
  const float *S, *gair, *gself, *elow, *nair, *delta;
  const int *iso; // jointMolIso / 100
  int64_t n;
  const double *S64 = nullptr;    // optional double overrides of S and gamma_air
  const double *gair64 = nullptr; // (set by marfa_ctx_set_line_params)
};

struct PrepParams {
  DeviceLines lines;
  const double *tips; // [n_iso][n_temp]
  int n_iso, n_temp;
  TipsGrid tgrid;     // temperature grid of the table
  const LevelConst *lv; // [Lc]
  int n_levels;         // Lc
  Consts c;
  double sscale;        // 2^scale_exp for the FP32-compensated hot records
  double *nus;          // [Lc][N]
  LineGen *gen;         // [Lc][N]
  Hot32 *hot32;         // [Lc][N] or null
  Hot64 *hot64;         // [Lc][N] or null
  int *err;             // device error word (max of status codes)
};

struct SortParams {
  const double *nu;     // unshifted, sorted
  const double *nus;    // [Lc][N]
  const double *margin; // [Lc] half-width of the re-ordering window
  int64_t n;
  int n_levels;
  int64_t *rank;        // [Lc][N] scratch
  double *snu;          // [Lc][N] sorted shifted centres
  int *sidx;            // [Lc][N] line index of each sorted slot
};

struct WindowTable {
  const double *sub_s, *sub_e;   // [n_sub] subinterval start / end
  const int64_t *lo, *hi;        // [n_sub] line window [lo, hi) (0-based)
  int n_sub;
};

struct FarParams {
  const double *nus;
  const Hot32 *hot32;
  const Hot64 *hot64;
  const LineGen *gen;
  const LevelConst *lv;
  WindowTable win;
  const int *chunk_sub;          // [C]
  const int64_t *chunk_begin, *chunk_end;
  int n_chunks;                  // C (per level)
  int n_levels;                  // Lc
  int64_t n_lines;
  double cutoff;
  double sscale;
  int shape;
  Consts c;
  double *out;                   // [Lc][C][NFAR]
};

// Rows of the fine kernel's slot buffer (values per staged line: ten on
// grids 1..9, fifteen in the finest-point pass).
constexpr int NSLOT = 15;

struct FineParams {
  const double *snu;
  const int *sidx;
  const LineGen *gen;
  const LevelConst *lv;
  WindowTable win;
  int64_t n_lines;
  int unit0;                     // first (level-in-chunk * n_sub + sub) of this batch
  int n_units;
  double cutoff;
  double sscale;
  int shape;
  Consts c;
  void *scratch;                 // [n_units][SCR_STRIDE] float or double
  int smem_cap;                  // near lines staged in shared memory
  void *gstage;                  // global staging for units above smem_cap
  int gstage_cap;                // lines per block in gstage
  size_t gstage_bytes;           // bytes per block in gstage
  int *err;
  int *queue;                    // work-queue head (zero before the launch)
  const int *order;              // optional processing order of the units
  void *vbuf;                    // per-block slot buffers in global memory
  size_t vbuf_stride;            // elements per block
  int vbuf_cap;                  // lines per slot row in vbuf
  int grid;                      // persistent blocks
  size_t smem_room;              // dynamic shared memory of the launch (bytes): a unit keeps its
                                 // slot rows there when they fit beside its staged lines
  int coop_k;                    // grids 1..coop_k: lane groups per cell pair in the site half
  int block_threads;             // threads per block (fine_block_threads)
};

struct CascadeParams {
  const void *scratch;           // from the fine kernel
  const double *far;             // [Lc][C][NFAR]
  const double *fold;            // [Lc][n_sub][NFAR] far sums per unit, or null (summed from far)
  const int *sub_chunk0;         // [n_sub + 1] first chunk of each subinterval
  const LevelConst *lv;
  int n_chunks, n_sub;
  int unit0, n_units;
  int level_out0;                // global level index of level-in-chunk 0
  double inv_sscale;
  int target;
  float *out;                    // [levels][n_sub][NT]
  double *out64;                 // optional
  double *dump;                  // optional raw-accumulator dump of one unit
  int dump_unit;
};

struct CountParams {
  const double *nus;
  WindowTable win;
  const int *chunk_sub;
  const int64_t *chunk_begin, *chunk_end;
  int n_chunks, n_levels;
  int64_t n_lines;
  double cutoff;
  unsigned long long *out;       // [Lc][C]
};

// ------------------------------------------------------------ adjoint
// Partial derivatives of the per-(level, line) spectroscopy.
struct LineAux {
  double ratio;    // S(T) / S_ref
  double dlnS_dT;  // d ln S(T) / dT
  double dg_dT;    // d gamma_L / dT (pself grows with T at fixed density)
  double dg_dP;    // d gamma_L / dP
  double dg_dgair; // d gamma_L / d gamma_air
  double delta;    // pressure shift: d nu' / dP
};

struct AdjPrepParams {
  DeviceLines lines;
  const double *tips;
  int n_iso, n_temp;
  TipsGrid tgrid;
  const LevelConst *lv;
  int n_levels;
  Consts c;
  LineAux *aux;                  // [Lc][N]
};

struct CascadeAdjParams {
  const double *scratch;         // FP64 accumulators of the batch
  const double *far;             // [Lc][C][NFAR]
  const double *fold;            // [Lc][n_sub][NFAR] far sums per unit, or null
  const int *sub_chunk0;
  const LevelConst *lv;
  int n_chunks, n_sub;
  int unit0, n_units;
  int level_out0;
  int target;
  const double *cot;             // [levels][n_sub][NT] cotangent of the records
  double *gscratch;              // [n_units][SCR_STRIDE] dL / d accumulator
};

struct AdjointParams {
  const double *snu;
  const int *sidx;
  const double *nus;
  const LineGen *gen;
  const LineAux *aux;
  const LevelConst *lv;
  WindowTable win;
  const int *sub_chunk0;
  const int64_t *chunk_begin, *chunk_end;
  int max_chunks;                // most far-kernel chunks of one subinterval
  int64_t n_lines;
  int unit0, n_units;
  int level_out0;
  double cutoff;
  Consts c;
  const double *gscratch;
  double *dS, *dgair;            // [N] per-line gradients (accumulated)
  double *dT, *dP;               // [levels]
};

// launchers (marfa_adjoint.cu)
cudaError_t launch_adjoint_prep(const AdjPrepParams &p, cudaStream_t st);
cudaError_t launch_cascade_adjoint(const CascadeAdjParams &p, cudaStream_t st);
cudaError_t launch_line_adjoint(const AdjointParams &p, int chi, int near_blocks, cudaStream_t st);

// launchers (marfa_kernels.cu)
cudaError_t launch_prep(const PrepParams &p, cudaStream_t st);
cudaError_t launch_sort(const SortParams &p, cudaStream_t st);
cudaError_t launch_far(const FarParams &p, int precision, int chi, cudaStream_t st);
// far-kernel partials summed per (level, subinterval, grid-0 position) over
// the subinterval's chunks, in chunk order: fold[Lc][n_sub][NFAR]
cudaError_t launch_far_fold(const double *far, const int *sub_chunk0, int n_chunks, int n_sub, int n_levels,
                            double *fold, cudaStream_t st);
cudaError_t launch_fine(const FineParams &p, int precision, int chi, cudaStream_t st);
cudaError_t launch_near_count(const FineParams &p, int *counts, cudaStream_t st);
// shared memory of `cap` staged lines and `rows` slot-buffer rows of `cap`
// values
size_t fine_smem_bytes(int cap, bool f64, int rows = 0);
size_t fine_vbuf_elems(int cap);
// block size of the fine kernel for a batch whose units have at most
// `max_near` near lines (small blocks below `small_below` lines; pair != 0:
// FP32c dense units on two 512-thread blocks per SM instead of one of 1024)
int fine_block_threads(int precision, int max_near, int small_below, int pair);
// most near lines a block of `threads` stages in shared memory (the opt-in
// limit minus the kernel's static shared memory)
cudaError_t fine_smem_lines(int precision, int chi, int threads, int *lines);
// dynamic shared memory of the launch and the persistent grid size: the whole
// per-block room for the large blocks, `smem_cap` lines (with slot rows when
// they fit) for the small ones
cudaError_t fine_plan(int precision, int chi, int threads, int smem_cap, size_t *smem_room, int *blocks);
cudaError_t launch_cascade(const CascadeParams &p, int precision, cudaStream_t st);
cudaError_t launch_count(const CountParams &p, cudaStream_t st);

} // namespace marfa
