// marfa_windows.h -- line windows of the subintervals, shared by the regular
// and the allocation-free entry points.
#pragma once
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <iterator>
#include <vector>
#include "marfa_gpu.h"

namespace marfa {

// Shifted-free centre nu of the 36-byte records as a random-access sequence
// (the records are packed, so nu is read byte-wise).
struct RecordNu {
  using iterator_category = std::random_access_iterator_tag;
  using value_type = double;
  using difference_type = std::ptrdiff_t;
  using pointer = const double *;
  using reference = double;
  const marfa_line_record *r;
  double operator*() const {
    double v;
    std::memcpy(&v, &r->nu, sizeof v);
    return v;
  }
  double operator[](difference_type i) const { return *(*this + i); }
  RecordNu &operator++() { ++r; return *this; }
  RecordNu operator++(int) { RecordNu t = *this; ++r; return t; }
  RecordNu &operator--() { --r; return *this; }
  RecordNu &operator+=(difference_type d) { r += d; return *this; }
  RecordNu &operator-=(difference_type d) { r -= d; return *this; }
  RecordNu operator+(difference_type d) const { return RecordNu{r + d}; }
  RecordNu operator-(difference_type d) const { return RecordNu{r - d}; }
  difference_type operator-(const RecordNu &o) const { return r - o.r; }
  bool operator==(const RecordNu &o) const { return r == o.r; }
  bool operator!=(const RecordNu &o) const { return r != o.r; }
  bool operator<(const RecordNu &o) const { return r < o.r; }
};

// Windows [lo, hi) of the first nsub subintervals of a run starting at
// start_wv; returns 0 or MARFA_E_DB with `bad` = the subinterval whose scan
// ran off the end (-1: before the starting line).  nu: the sorted centres
// (a random-access sequence of doubles).
//   determineStartingSpectralLine (main.f90:196-248): the first record with
//   nu > start - cutoff, when start > cutoff.
//   SUBINTERVALS_LOOP with the lblScheme window recurrence (LBL.f90:41-61,
//   main.f90:138-144): the scan from line_idx stops at the first nu >=
//   start + 10 + cutoff; the next window starts at the last scanned line
//   with nu <= capWV = max(start - cutoff + 10, starting line), or stays.
// The list is sorted, so the reference's linear scans are binary searches
// here, with the same results.
template <class It>
int plan_windows_of(It nu, int64_t n, double start_wv, int nsub, double cut, std::vector<double> &ss,
                    std::vector<double> &se, std::vector<int64_t> &lo, std::vector<int64_t> &hi, int &bad) {
  bad = -1;
  int64_t start_idx = 0;
  double start_line = nu[0];
  if (start_wv > cut) {
    const double ext = start_wv - cut;
    start_idx = std::upper_bound(nu, nu + n, ext) - nu;
    if (start_idx >= n) return MARFA_E_DB;
    start_line = nu[start_idx];
  }
  int64_t line_idx = start_idx;
  double s = start_wv;
  for (int isub = 0; isub < nsub; ++isub) {
    const double ext_end = s + 10.0 + cut;
    double cap = (s - cut) + 10.0;
    if (cap <= start_line) cap = start_line;
    const int64_t I = std::lower_bound(nu + line_idx, nu + n, ext_end) - nu;
    if (I >= n) {
      bad = isub;
      return MARFA_E_DB;
    }
    const int64_t last = (std::upper_bound(nu + line_idx, nu + I, cap) - nu) - 1;
    const int64_t next = last >= line_idx ? last : line_idx;
    ss.push_back(s);
    se.push_back(s + 10.0);
    lo.push_back(line_idx);
    hi.push_back(I);
    line_idx = next;
    s = s + 10.0;
  }
  return MARFA_OK;
}

} // namespace marfa
