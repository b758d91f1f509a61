// lmc_internal.h -- shared host-side helpers of libluminis_b200 (not installed).
#pragma once
#include <complex>
#include <cstdio>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "luminis_b200.h"

namespace lmc {

// An NVTX range named `name` for the object's lifetime (scene set-up, launches, tally
// read-back), so a profiler that traces NVTX shows the host phases of a run beside its
// kernels.  Without a profiler attached each push/pop is a branch on a null callback.
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

// Thread-local last-error message behind lmc_last_error().
std::string &last_error();

inline lmc_status fail(lmc_status code, const char *msg)
{
  last_error() = msg;
  return code;
}

inline lmc_status fail(lmc_status code, const std::string &msg)
{
  last_error() = msg;
  return code;
}

// The Mie series of one size parameter in the form the angular sums consume:
// ap[n-1] = (2n+1)/(n(n+1)) (a_n + b_n), bp[n-1] = (2n+1)/(n(n+1)) (a_n - b_n), or the
// small-particle limit's three coefficients (ntrm == 0).  Same numbers as the per-angle
// evaluation in lmc_mie / lmc_amplitude_table / lmc_sampling_table.
struct MieSeries {
  int ntrm = 0;
  bool conj_out = false;
  double small_rtmp = 0.0;
  std::complex<double> small_a1, small_a2, small_b1;
  std::vector<std::complex<double>> ap, bp;
  double qsca = 0.0;
};

bool mie_series(double x, double m_re, double m_im, MieSeries &out);

// Device buffer -> pageable host buffer through two pinned 16 MiB halves shared by the
// process, host-thread copies overlapping the DMA; `stream` is a cudaStream_t.  Blocks
// until the copy is done.
lmc_status read_back(double *h_dst, const double *d_src, size_t bytes, void *stream);

}  // namespace lmc
