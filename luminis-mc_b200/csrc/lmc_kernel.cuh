// lmc_kernel.cuh -- device code of the photon-propagation kernel (sm_100a).
//
// One persistent kernel replaces run_simulation_parallel's worker pool and
// run_photon (src/simulation.cpp:105-617).  Each thread owns one photon at a
// time and advances it ONE scattering event per loop iteration; a thread whose
// photon died takes the next photon index in the same iteration (warp-
// aggregated atomic on a global counter), so the 32 lanes of a warp keep doing
// events instead of idling until the warp's longest path ends.  Each photon
// draws from its own Philox4x32-10 stream keyed by (seed, photon index) in the
// reference's draw order, so results do not depend on the launch shape, as the
// reference's do not depend on n_threads.
//
// State layout: what every event reads lives in registers (position, frame,
// Jones vector, weight, the running interior Jones product, the previous frame
// and position); what only a CBS detection reads -- the first-scatter frame and
// position and the newest event's raw Jones factors -- lives in shared memory,
// one slot per thread.  The emission time is recomputed from the counter-based
// stream when a detector needs it instead of being carried.
//
// Precision: `R` is the transport type (float or double).  The weight, the
// geometric path length, the CBS geometric phase k (s_out + s_in).(r_n - r_1)
// and every tally are binary64 in both modes.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "lmc_device.cuh"
#include "luminis_b200.h"

namespace lmc {
namespace dev {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kBlock = 256;                 // threads per block (upper bound)

// ------------------------------------------------------------------ math by type
__device__ __forceinline__ float m_log(float x) { return logf(x); }
__device__ __forceinline__ double m_log(double x) { return log(x); }
__device__ __forceinline__ float m_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double m_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float m_atan2(float y, float x) { return atan2f(y, x); }
__device__ __forceinline__ double m_atan2(double y, double x) { return atan2(y, x); }
__device__ __forceinline__ void m_sincos(float x, float *s, float *c) { sincosf(x, s, c); }
__device__ __forceinline__ void m_sincos(double x, double *s, double *c) { sincos(x, s, c); }
__device__ __forceinline__ void m_sincospi(float x, float *s, float *c) { sincospif(x, s, c); }
// sin and cos of 2 pi u for u in [0, 1] in binary32, for the azimuth trials: u is
// reduced to the nearest quarter turn, r = 4u - rint(4u) in [-1/2, 1/2] (exact for
// the u24 values), and sin / cos of a = r pi / 2 (|a| <= pi / 4) are their Taylor
// series to degree 9 / 10 (truncation < 2e-9, below binary32 rounding); the quarter
// turns then rotate the pair.  Shorter than the general sincospif, whose argument
// range the trials do not need.
__device__ __forceinline__ void sincos_turn(float u, float *s, float *c)
{
  const float x4 = 4.0f * u;
  const float q = rintf(x4);
  const float a = (x4 - q) * 1.5707963267948966f;
  const float a2 = a * a;
  float sp = fmaf(a2, 2.7557319223985893e-6f, -1.9841269841269841e-4f);
  sp = fmaf(a2, sp, 8.3333333333333333e-3f);
  sp = fmaf(a2, sp, -1.6666666666666667e-1f);
  const float sa = fmaf(a * a2, sp, a);
  float cp = fmaf(a2, -2.7557319223985891e-7f, 2.4801587301587302e-5f);
  cp = fmaf(a2, cp, -1.3888888888888889e-3f);
  cp = fmaf(a2, cp, 4.1666666666666667e-2f);
  cp = fmaf(a2, cp, -0.5f);
  const float ca = fmaf(a2, cp, 1.0f);
  const int qi = ((int)q) & 3;
  const float ss = (qi & 1) ? ca : sa, cc = (qi & 1) ? sa : ca;
  *s = (qi & 2) ? -ss : ss;
  *c = ((qi + 1) & 2) ? -cc : cc;
}
__device__ __forceinline__ void m_sincos_turn(float u, float *s, float *c) { sincos_turn(u, s, c); }
__device__ __forceinline__ void m_sincos_turn(double u, double *s, double *c) { sincospi(2.0 * u, s, c); }
__device__ __forceinline__ void m_sincospi(double x, double *s, double *c) { sincospi(x, s, c); }
__device__ __forceinline__ float m_nudge(float z, float zi, bool up)
{
  // The reference nudges by 1e-12 (src/simulation.cpp:351-352); in binary32 that
  // is below one ulp of z for z > ~1e-5, so step to the adjacent float instead.
  return (z != zi) ? z : nextafterf(zi, up ? INFINITY : -INFINITY);
}
__device__ __forceinline__ double m_nudge(double z, double, bool) { return z; }

// Smallest norm the reference still divides by (1e-300, src/detector.cpp:1152,
// src/simulation.cpp:557); the binary32 path uses the nearest normal float.
template <typename R> __device__ __forceinline__ R tiny();
template <> __device__ __forceinline__ float tiny<float>() { return 1e-37f; }
template <> __device__ __forceinline__ double tiny<double>() { return 1e-300; }

template <typename R> struct Cx {
  R re, im;
};
template <typename R> __device__ __forceinline__ Cx<R> cmul(Cx<R> a, Cx<R> b)
{
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R> __device__ __forceinline__ Cx<R> cadd(Cx<R> a, Cx<R> b) { return {a.re + b.re, a.im + b.im}; }
template <typename R> __device__ __forceinline__ Cx<R> cscale(Cx<R> a, R s) { return {a.re * s, a.im * s}; }
template <typename R> __device__ __forceinline__ R cnorm(Cx<R> a) { return a.re * a.re + a.im * a.im; }

// scalar fields by transport type
template <typename R> __device__ __forceinline__ R med_mfp(const Medium &m);
template <> __device__ __forceinline__ float med_mfp<float>(const Medium &m) { return m.mfp_f; }
template <> __device__ __forceinline__ double med_mfp<double>(const Medium &m) { return m.mfp; }
template <typename R> __device__ __forceinline__ R med_mut(const Medium &m);
template <> __device__ __forceinline__ float med_mut<float>(const Medium &m) { return m.mu_t_f; }
template <> __device__ __forceinline__ double med_mut<double>(const Medium &m) { return m.mu_t; }
template <typename R> __device__ __forceinline__ R lay_mfp(const Layer &l);
template <> __device__ __forceinline__ float lay_mfp<float>(const Layer &l) { return l.mfp_f; }
template <> __device__ __forceinline__ double lay_mfp<double>(const Layer &l) { return l.mfp; }
template <typename R> __device__ __forceinline__ R lay_mut(const Layer &l);
template <> __device__ __forceinline__ float lay_mut<float>(const Layer &l) { return l.mu_t_f; }
template <> __device__ __forceinline__ double lay_mut<double>(const Layer &l) { return l.mu_t; }
template <typename R> __device__ __forceinline__ R sc_iface(const Scene &s, int i);
template <> __device__ __forceinline__ float sc_iface<float>(const Scene &s, int i) { return s.interfaces_f[i]; }
template <> __device__ __forceinline__ double sc_iface<double>(const Scene &s, int i) { return s.interfaces[i]; }
template <typename R> __device__ __forceinline__ R sc_plane(const Scene &s, int i);
template <> __device__ __forceinline__ float sc_plane<float>(const Scene &s, int i) { return s.plane_z_f[i]; }
template <> __device__ __forceinline__ double sc_plane<double>(const Scene &s, int i) { return s.plane_z[i]; }
template <typename R> __device__ __forceinline__ R sc_top(const Scene &s);
template <> __device__ __forceinline__ float sc_top<float>(const Scene &s) { return s.top_f; }
template <> __device__ __forceinline__ double sc_top<double>(const Scene &s) { return s.top; }

// ------------------------------------------------------------------------ RNG
// Philox4x32-10 (Salmon et al., SC'11); stream contract in luminis_b200.h.
// A photon's stream is generated a Philox block (4 words) at a time into a ring of
// kRing words; draw d reads word d (u24) or words 2d, 2d+1 (u53).  The transport
// kernel keeps the ring in shared memory (one column per thread) and tops it up at
// the top of every event, where the warp is converged, so the azimuth rejection
// loop -- whose trial count differs from lane to lane -- finds its numbers already
// generated instead of running the ten Philox rounds with a few lanes active.
constexpr uint32_t kRing = 16;

template <int kStride> struct RngT {
  uint32_t p_lo, p_hi;
  uint32_t draw;               // draws consumed (stream position)
  uint32_t filled;             // words generated so far (a multiple of 4)
  uint32_t *ring;              // kRing words, kStride apart
  __device__ __forceinline__ uint32_t &word(uint32_t w) const
  {
    return ring[(w & (kRing - 1u)) * kStride];
  }
};
using Rng = RngT<kBlock>;

// The ten rounds of one block, inlined where the ring is filled: at the once-per-event
// prefetch and at a draw that finds the ring dry.
__device__ __forceinline__ uint4 philox_block(uint32_t block, uint32_t p_lo, uint32_t p_hi,
                                              uint32_t key0, uint32_t key1)
{
  uint32_t c0 = block, c1 = 0u, c2 = p_lo, c3 = p_hi;
  uint32_t k0 = key0, k1 = key1;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
    const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return make_uint4(c0, c1, c2, c3);
}

// Words per draw: u24 takes one 32-bit word, u53 two.  binary32 transport always
// draws u24; binary64 transport draws u53, or u24 when the run asks for it (the
// same numbers as a binary32 run, to measure precision alone).
template <typename R> __device__ __forceinline__ uint32_t words_per_draw(const RunParams &rp);
template <> __device__ __forceinline__ uint32_t words_per_draw<float>(const RunParams &) { return 1u; }
template <> __device__ __forceinline__ uint32_t words_per_draw<double>(const RunParams &rp)
{
  return rp.stream_u24 ? 1u : 2u;
}

template <int S> __device__ __forceinline__ void rng_reset(RngT<S> &g, unsigned long long index)
{
  g.p_lo = (uint32_t)index;
  g.p_hi = (uint32_t)(index >> 32);
  g.draw = 0;
  g.filled = 0;
}

// Generate the next block into the ring (words filled .. filled + 3).
template <int S> __device__ __forceinline__ void rng_fill(RngT<S> &g, const RunParams &rp)
{
  const uint4 b = philox_block(g.filled >> 2, g.p_lo, g.p_hi, rp.key0, rp.key1);
  g.word(g.filled) = b.x;
  g.word(g.filled + 1u) = b.y;
  g.word(g.filled + 2u) = b.z;
  g.word(g.filled + 3u) = b.w;
  g.filled += 4u;
}

// Top the ring up (call while converged): up to two blocks, as long as a whole
// block fits behind the words not yet consumed.
template <typename R, int S> __device__ __forceinline__ void rng_prefetch(RngT<S> &g, const RunParams &rp)
{
  const uint32_t used = g.draw * words_per_draw<R>(rp);
#pragma unroll 1
  for (int i = 0; i < 2; ++i)
    if (g.filled + 4u <= used + kRing)
      rng_fill(g, rp);
}

// Words of the next draw; generates a block only if the ring ran dry.
template <typename R, int S> __device__ __forceinline__ void rng_words(RngT<S> &g, const RunParams &rp,
                                                                       uint32_t &lo, uint32_t &hi)
{
  const uint32_t wpd = words_per_draw<R>(rp);
  const uint32_t w0 = g.draw * wpd;
  if (w0 + wpd > g.filled)
    rng_fill(g, rp);
  lo = g.word(w0);
  hi = wpd == 2u ? g.word(w0 + 1u) : 0u;
  g.draw++;
}

// The uniform value of a draw's word(s): "u24" (2 (x >> 9) + 1) 2^-24 or "u53"
// (2 (w >> 12) + 1) 2^-53 of the 64-bit word hi:lo; binary64 on the u24 stream
// returns exactly the binary32 run's value.
template <typename R> __device__ __forceinline__ R words_uniform(const RunParams &rp, uint32_t lo, uint32_t hi);
template <> __device__ __forceinline__ float words_uniform<float>(const RunParams &, uint32_t w, uint32_t)
{
  return __uint2float_rn(2u * (w >> 9) + 1u) * 5.9604644775390625e-8f;   // 2^-24
}
template <> __device__ __forceinline__ double words_uniform<double>(const RunParams &rp, uint32_t lo, uint32_t hi)
{
  if (rp.stream_u24)
    return (double)(__uint2float_rn(2u * (lo >> 9) + 1u) * 5.9604644775390625e-8f);
  const unsigned long long w = ((unsigned long long)hi << 32) | lo;
  return __ull2double_rn(2ull * (w >> 12) + 1ull) * 1.1102230246251565e-16;   // 2^-53
}

template <typename R, int S> __device__ __forceinline__ R uniform(RngT<S> &g, const RunParams &rp)
{
  uint32_t lo, hi;
  rng_words<R>(g, rp, lo, hi);
  return words_uniform<R>(rp, lo, hi);
}

// Draw g.draw + k without consuming it; the caller has checked that the ring holds it.
template <typename R, int S> __device__ __forceinline__ R peek_uniform(const RngT<S> &g, const RunParams &rp,
                                                                       uint32_t k)
{
  const uint32_t wpd = words_per_draw<R>(rp);
  const uint32_t w0 = (g.draw + k) * wpd;
  return words_uniform<R>(rp, g.word(w0), wpd == 2u ? g.word(w0 + 1u) : 0u);
}

// --------------------------------------------------------------------- photon
template <typename R> struct Photon {
  R px, py, pz;
  R P[9];                      // rows m, n, s of P_local (photon.hpp:117)
  Cx<R> Em, En;                // Jones vector in (m, n)
  double w;                    // weight: binary64 (thousands of products per path)
  double opath;                // geometric path length (time): binary64
  R pen;                       // penetration depth (records only)
  uint32_t events;
  int layer, last_med;
  int scene;                   // sweep: the photon's scene
  Rng rng;
  __device__ __forceinline__ unsigned long long index() const
  {
    return ((unsigned long long)rng.p_hi << 32) | rng.p_lo;
  }
};

// Per-thread CBS state, in shared memory (one column per thread): the reverse
// path reads it only at a detection, and keeping it out of registers lets more
// warps share an SM.  Lives in dynamic shared memory (the binary64 layout exceeds
// the 48 KB static limit).
template <typename R> struct Side {
  uint32_t ring[kRing][kBlock];  // the photon's generated Philox words (see RngT)
  int first_med[kBlock];
  // the reverse-path history from here on (a launch that replays it instead allocates
  // only the members above: side_slim_bytes)
  R first[12][kBlock];         // r_1 (3), then P1 rows m_1, n_1, s_1 (9)
  R last[6][kBlock];           // S2, S1 (re, im) and cos, sin(phi) of the newest scatter
  R ang[4][kBlock];            // cos, sin theta and cos, sin phi of the newest scatter:
                               // P_{n-1} = A^T P_n when a hit needs it (prev_frame)
  R rn[3][kBlock];             // position of the newest scatter (r_n)
  R T[8][kBlock];              // matrix_T_raw: normalised interior Jones product (re, im)
};

// Dynamic shared memory of a transport block: the Side arrays, then (kAdj) the
// likelihood-ratio scores, adj_K * kBlock R, or (estimator kernels) the block's copies
// of the estimated grids, RunParams::est_smem_doubles doubles.
template <typename R> __host__ __device__ constexpr size_t side_bytes()
{
  return (sizeof(Side<R>) + 15) & ~size_t(15);
}
// The ring and the first species alone: a transport launch without reverse-path
// bookkeeping (rp.track_reverse == 0) touches nothing else of Side.
template <typename R> __host__ __device__ constexpr size_t side_slim_bytes()
{
  return (sizeof(uint32_t) * kRing * kBlock + sizeof(int) * kBlock + 15) & ~size_t(15);
}

struct Counters {
  uint32_t events, steps, draws;
};

// ------------------------------------------------------- likelihood-ratio score
// Score of a photon history: d/d(param) of log(path density x weight), summed over
// its free flights, albedo factors and HG angle draws (the estimator of
// oracle/lmc_oracle.c, in the same order of operations).  A free flight from medium
// a draws tau ~ Exp(1), step = mfp_a tau, and every interface rescales the remaining
// distance by mu_t_old / mu_t_new (src/simulation.cpp:318-382): its optical depth
// O = sum_i d_i mu_t_i is exponential with mean m_a = mfp_a mu_t_a.  A flight ending
// in a scatter in medium c has log density log mu_t_c - log m_a - O / m_a; one cut
// by a sensor hit has log survival -O / m_a.  Parameters k = 4 medium + (mu_a, mu_s,
// mfp, g).  The running scores live in shared memory, one column per thread.
template <typename R> __device__ __forceinline__ R med_mus(const Medium &m);
template <> __device__ __forceinline__ float med_mus<float>(const Medium &m) { return m.mu_s_f; }
template <> __device__ __forceinline__ double med_mus<double>(const Medium &m) { return m.mu_s; }
template <typename R> __device__ __forceinline__ R med_g(const Medium &m);
template <> __device__ __forceinline__ float med_g<float>(const Medium &m) { return m.hg_g_f; }
template <> __device__ __forceinline__ double med_g<double>(const Medium &m) { return m.hg_g; }

template <typename R> struct Flight {
  R *score;                    // this thread's column: score[k * kBlock]
  R m, O, seg_len;             // m_a; depth of completed segments; current segment length
  int a, cross, seg_med;       // start medium; crossed an interface; current segment's medium
  __device__ __forceinline__ R &operator[](int k) const { return score[k * kBlock]; }
};

template <typename R>
__device__ __forceinline__ void flight_start(const Scene &sc, Flight<R> &f, int med)
{
  const Medium &m = sc.media[med];
  f.a = med;
  f.m = med_mfp<R>(m) * med_mut<R>(m);
  f.O = R(0);
  f.cross = 0;
}

template <typename R>
__device__ __forceinline__ void flight_segment_done(const Scene &sc, Flight<R> &f, int med, R d)
{
  f[4 * med + 0] -= d / f.m;
  f[4 * med + 1] -= d / f.m;
  f.O += d * med_mut<R>(sc.media[med]);
  f.cross = 1;
}

template <typename R>
__device__ __forceinline__ void flight_scatter(const Scene &sc, Flight<R> &f, int c, R d)
{
  const int a = f.a;
  const R mfp_a = med_mfp<R>(sc.media[a]);
  if (!f.cross) {
    f[4 * a + 2] += (d / mfp_a - R(1)) / mfp_a;
    return;
  }
  const R mt_a = med_mut<R>(sc.media[a]), mt_c = med_mut<R>(sc.media[c]);
  f[4 * c + 0] -= d / f.m;
  f[4 * c + 1] -= d / f.m;
  const R O = f.O + d * mt_c;
  f[4 * c + 0] += R(1) / mt_c;
  f[4 * c + 1] += R(1) / mt_c;
  f[4 * a + 0] += O / (f.m * mt_a) - R(1) / mt_a;
  f[4 * a + 1] += O / (f.m * mt_a) - R(1) / mt_a;
  f[4 * a + 2] += O / (mfp_a * f.m) - R(1) / mfp_a;
}

// Albedo and HG terms of a scatter in medium c with sampled cos(theta).
template <typename R>
__device__ __forceinline__ void flight_event(const Scene &sc, Flight<R> &f, int c, R cos_theta)
{
  const Medium &m = sc.media[c];
  const R mt = med_mut<R>(m);
  if (mt > R(0)) {
    f[4 * c + 0] += R(-1) / mt;
    f[4 * c + 1] += R(1) / med_mus<R>(m) - R(1) / mt;
  }
  if (m.theta_kind == LMC_THETA_HG) {
    const R g = med_g<R>(m);
    f[4 * c + 3] += R(-2) * g / (R(1) - g * g) -
                    R(3) * (g - cos_theta) / (R(1) + g * g - R(2) * g * cos_theta);
  }
}

// Score k of a sensor crossing at fraction t of the current segment.
template <typename R>
__device__ __forceinline__ R flight_hit_score(const Scene &sc, const Flight<R> &f, R t, int k)
{
  R v = f[k];
  const R d = t * f.seg_len;
  const int a = f.a;
  const R mfp_a = med_mfp<R>(sc.media[a]);
  if (!f.cross) {
    if (k == 4 * a + 2)
      v += (d / mfp_a) / mfp_a;
    return v;
  }
  const int sm = f.seg_med;
  if (k == 4 * sm + 0 || k == 4 * sm + 1)
    v -= d / f.m;
  const R O = f.O + d * med_mut<R>(sc.media[sm]);
  if (k == 4 * a + 0 || k == 4 * a + 1)
    v += O / (f.m * med_mut<R>(sc.media[a]));
  if (k == 4 * a + 2)
    v += O / (mfp_a * f.m);
  return v;
}

template <typename R> __device__ __forceinline__ int layer_index_at(const Scene &sc, R z)
{                                                          // src/sample.cpp:221-235
  if (z < R(0))
    return sc.n_layers;
  if (!sc.top_is_inf && z >= sc_top<R>(sc))
    return sc.n_layers;
  int idx = 0;
  for (int i = 0; i < sc.n_interfaces; ++i)
    idx += (sc_iface<R>(sc, i) <= z) ? 1 : 0;              // upper_bound on a sorted list
  return idx < sc.n_layers ? idx : sc.n_layers;
}

template <typename R>
__device__ __forceinline__ bool find_next_interface(const Scene &sc, R zc, R zt, R &out)
{                                                          // src/sample.cpp:237-266
  if (zt > zc) {
    for (int i = 0; i < sc.n_interfaces; ++i) {
      const R zi = sc_iface<R>(sc, i);
      if (zi > zc) {
        if (zi <= zt) {
          out = zi;
          return true;
        }
        return false;
      }
    }
  } else if (zt < zc) {
    for (int i = sc.n_interfaces - 1; i >= 0; --i) {
      const R zi = sc_iface<R>(sc, i);
      if (zi < zc) {
        if (zi >= zt) {
          out = zi;
          return true;
        }
        return false;
      }
    }
  }
  return false;
}

// ---------------------------------------------------------------- theta sampling
// SamplingTable::Sample (src/table.cpp:50-66) with a guide table that narrows
// std::lower_bound's range; the index found is the same.
__device__ __forceinline__ double table_sample_f64(const Medium &m, double u)
{
  int j = (int)(u * (double)kGuideBuckets);
  if (!in_bounds(kBoundGuide, j >= 0 && j < kGuideBuckets))
    j = j < 0 ? 0 : kGuideBuckets - 1;
  int lo = __ldg(m.guide_d + j), hi = __ldg(m.guide_d + j + 1);
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(m.th_cdf_d + mid) < u)
      lo = mid + 1;
    else
      hi = mid;
  }
  if (!in_bounds(kBoundCdf, lo >= 0 && lo < m.theta_n))
    lo = lo < 0 ? 0 : m.theta_n - 1;
  if (lo == 0)
    return __ldg(m.th_val_d);
  const double c0 = __ldg(m.th_cdf_d + lo - 1), c1 = __ldg(m.th_cdf_d + lo);
  const double v0 = __ldg(m.th_val_d + lo - 1), v1 = __ldg(m.th_val_d + lo);
  const double t = (u - c0) / (c1 - c0);
  return v0 + t * (v1 - v0);
}

// The binary32 path searches the same binary64 CDF: near cdf = 1 a binary32 CDF
// keeps only ~6e-8 of resolution, coarser than the increments of low-probability
// (back-scatter) bins.  u24 values are exact in binary64, so the search finds the
// reference's index; the lerp uses a precomputed slope per node.
__device__ __forceinline__ double table_sample_f32(const Medium &m, float u)
{
  const double ud = u;
  int j = (int)(u * (float)kGuideBuckets);
  if (!in_bounds(kBoundGuide, j >= 0 && j < kGuideBuckets))
    j = j < 0 ? 0 : kGuideBuckets - 1;
  int lo = __ldg(m.guide_d + j), hi = __ldg(m.guide_d + j + 1);
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(m.th_cdf_d + mid) < ud)
      lo = mid + 1;
    else
      hi = mid;
  }
  if (!in_bounds(kBoundCdf, lo >= 0 && lo < m.theta_n))
    lo = lo < 0 ? 0 : m.theta_n - 1;
  if (lo == 0)
    return __ldg(m.th_val_d);
  const double c0 = __ldg(m.th_cdf_d + lo - 1);
  const double slope = __ldg(&m.th_cs[lo].y);
  return __ldg(m.th_val_d + lo - 1) + (ud - c0) * slope;
}

template <typename R> __device__ __forceinline__ R sample_theta(const Medium &m, R u);

template <> __device__ __forceinline__ float sample_theta<float>(const Medium &m, float u)
{
  if (m.theta_kind == LMC_THETA_HG) {                      // src/phase.cpp:108-115
    // Same inverse CDF written through 1 -/+ cos(theta) so that neither cancels:
    // 1 - c = (1-g)(1-u)(1-g+frac)/d, 1 + c = (1+g)u(1+g+frac)/d, d = 1-g+2gu,
    // theta = 2 atan2(sqrt(1-c), sqrt(1+c)); acos(c) loses all precision near c = 1.
    const float g = m.hg_g_f;
    const float d = 1.0f - g + 2.0f * g * u;
    const float frac = (1.0f - g * g) / d;
    const float omc = (1.0f - g) * (1.0f - u) * (1.0f - g + frac) / d;
    const float opc = (1.0f + g) * u * (1.0f + g + frac) / d;
    return 2.0f * atan2f(sqrtf(omc), sqrtf(opc));
  }
  if (m.theta_kind == LMC_THETA_UNIFORM)
    return 2.0f * atan2f(sqrtf(1.0f - u), sqrtf(u));        // acos(2u - 1)
  const double v = table_sample_f32(m, u);
  if (m.theta_kind == LMC_THETA_TABLE)
    return (float)v;
  // cos-theta tables: theta = 2 atan2(sqrt(1 - c), sqrt(1 + c)) with 1 -/+ c formed
  // in binary64, accurate near c = +-1 where acosf of a rounded c is not
  return 2.0f * atan2f(sqrtf((float)(1.0 - v)), sqrtf((float)(1.0 + v)));
}

template <> __device__ __forceinline__ double sample_theta<double>(const Medium &m, double u)
{
  if (m.theta_kind == LMC_THETA_HG) {
    const double g = m.hg_g, gg = g * g;
    const double frac = (1.0 - gg) / (1.0 - g + 2.0 * g * u);
    // clamped: rounding can leave cos theta an ulp outside [-1, 1] near u -> 0, 1
    return acos(fmin(fmax((1.0 + gg - frac * frac) / (2.0 * g), -1.0), 1.0));
  }
  if (m.theta_kind == LMC_THETA_UNIFORM)
    return acos(2.0 * u - 1.0);
  const double v = table_sample_f64(m, u);
  return m.theta_kind == LMC_THETA_TABLE ? v : acos(v);
}

// DataTable::Sample on the uniform theta grid (src/table.cpp:100-118): S2, S1.
template <typename R> __device__ __forceinline__ void amplitudes(const Medium &m, R theta, Cx<R> &s2, Cx<R> &s1);

template <> __device__ __forceinline__ void amplitudes<float>(const Medium &m, float theta, Cx<float> &s2, Cx<float> &s1)
{
  const float pos = theta * m.amp_inv_dx_f;
  const int last = m.amp_n - 1;
  const float4 *st = m.amp_stage;        // the block's shared copy, when staged
  auto node = [&](int k) { return st ? st[k] : __ldg(m.amp_f + k); };
  float4 a;
  if (pos <= 0.0f) {
    a = node(0);
  } else if (pos >= (float)last) {
    a = node(last);
  } else {
    int i = (int)pos;
    if (!in_bounds(kBoundAmp, i >= 0 && i < last))
      i = i < 0 ? 0 : last - 1;
    const float t = pos - (float)i;
    const float4 y0 = node(i), y1 = node(i + 1);
    a = make_float4(y0.x + t * (y1.x - y0.x), y0.y + t * (y1.y - y0.y), y0.z + t * (y1.z - y0.z),
                    y0.w + t * (y1.w - y0.w));
  }
  s1 = {a.x, a.y};
  s2 = {a.z, a.w};
}

template <> __device__ __forceinline__ void amplitudes<double>(const Medium &m, double theta, Cx<double> &s2, Cx<double> &s1)
{
  const double pos = theta * m.amp_inv_dx;
  const int last = m.amp_n - 1;
  double4 a;
  if (pos <= 0.0) {
    a = m.amp_d[0];
  } else if (pos >= (double)last) {
    a = m.amp_d[last];
  } else {
    int i = (int)pos;
    if (!in_bounds(kBoundAmp, i >= 0 && i < last))
      i = i < 0 ? 0 : last - 1;
    const double t = pos - (double)i;
    const double4 y0 = m.amp_d[i], y1 = m.amp_d[i + 1];
    a = make_double4(y0.x + t * (y1.x - y0.x), y0.y + t * (y1.y - y0.y), y0.z + t * (y1.z - y0.z),
                     y0.w + t * (y1.w - y0.w));
  }
  s1 = {a.x, a.y};
  s2 = {a.z, a.w};
}

// ------------------------------------------------------------------ geometry
template <typename R> struct V3 {
  R x, y, z;
};
template <typename R> __device__ __forceinline__ V3<R> v3(R x, R y, R z) { return {x, y, z}; }
template <typename R> __device__ __forceinline__ R vdot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename R> __device__ __forceinline__ V3<R> vscale(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <typename R> __device__ __forceinline__ V3<R> vcross_unit(V3<R> a, V3<R> b)
{                                                          // src/vec.cpp:14-26 (normalises)
  V3<R> r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
  const R nf = m_sqrt(vdot(r, r));
  if (nf > R(0))
    r = vscale(r, R(1) / nf);
  return r;
}
template <typename R> __device__ __forceinline__ V3<R> safe_unit(V3<R> v, V3<R> fb)
{                                                          // src/utils.cpp:39-50
  const R eps = R(1e-20);
  const R n2 = vdot(v, v);
  if (n2 < eps) {
    const R f2 = vdot(fb, fb);
    if (f2 < eps)
      return v3<R>(R(1), R(0), R(0));
    return vscale(fb, R(1) / m_sqrt(f2));
  }
  return vscale(v, R(1) / m_sqrt(n2));
}
template <typename R> __device__ __forceinline__ V3<R> row(const R *P, int r) { return {P[3 * r], P[3 * r + 1], P[3 * r + 2]}; }

// Angle between unit vectors.  binary64 follows the reference,
// acos(clamp_pm1(a.b)) (src/detector.cpp:1098,1137); binary32 uses
// atan2(|a x b|, a.b), because acos of a dot product near +-1 is ill-conditioned.
__device__ __forceinline__ double unit_angle(V3<double> a, V3<double> b)
{
  double c = vdot(a, b);
  c = c > 1.0 ? 1.0 : (c < -1.0 ? -1.0 : c);
  return acos(c);
}
__device__ __forceinline__ float unit_angle(V3<float> a, V3<float> b)
{
  const float x = a.y * b.z - a.z * b.y, y = a.z * b.x - a.x * b.z, z = a.x * b.y - a.y * b.x;
  return atan2f(sqrtf(x * x + y * y + z * z), vdot(a, b));
}
// Exit polar angle theta = acos(-s_z) (src/detector.cpp:1273); binary32 uses
// atan2(sqrt(s_x^2 + s_y^2), -s_z), which resolves the small angles of the CBS cone.
__device__ __forceinline__ double exit_theta(double, double, double sz) { return acos(-sz); }
__device__ __forceinline__ float exit_theta(float sx, float sy, float sz)
{
  return atan2f(sqrtf(sx * sx + sy * sy), -sz);
}

// The exit direction as the sensors' angular tests read it.  Binary32 transport's
// direction drifts off unit length as a random walk of its roundings (|s| - 1 ~ 6e-8
// sqrt(events): ~6e-6 after 1e4 events), and a cosine test on a narrow cone (1 - cos 20
// mrad = 2e-4) turns that into lost hits at both edges (3.7 % of a 20 mrad cone's hits
// at 1.1e4 events per photon), so binary32 divides by |s| in binary64.  Binary64 keeps the
// reference's components as they are (|s| - 1 ~ 1e-15).
__device__ __forceinline__ void exit_dir(double sx, double sy, double sz, double *d)
{
  d[0] = sx; d[1] = sy; d[2] = sz;
}
__device__ __forceinline__ void exit_dir(float sx, float sy, float sz, double *d)
{
  const double x = sx, y = sy, z = sz;
  const double inv = 1.0 / sqrt(x * x + y * y + z * z);
  d[0] = x * inv; d[1] = y * inv; d[2] = z * inv;
}

// ---------------------------------------------------------------- source
// Laser::emit_photon's random part (src/laser.cpp:11-28, :42-75, :77-99): launch
// x, y and emission time, drawn from the photon's stream starting at draw 0.
template <typename R, int S>
__device__ void source_sample(const Laser &L, RngT<S> &g, const RunParams &rp, double &x, double &y,
                              double &t)
{
  x = L.pos[0];
  y = L.pos[1];
  if (L.source == 1) {
    const double th = (double)uniform<R>(g, rp) * 2.0 * 3.141592653589793;
    const double r = sqrt((double)uniform<R>(g, rp)) * L.sigma;
    x = x + r * cos(th);
    y = y + r * sin(th);
  } else if (L.source == 2) {
    for (int axis = 0; axis < 2; ++axis) {                 // Rng::normal, src/rng.cpp:18-27
      const double u1 = (double)uniform<R>(g, rp);         // never 0 in this stream
      const double u2 = (double)uniform<R>(g, rp);
      const double z0 = sqrt(-2.0 * log(u1)) * cos(2.0 * 3.141592653589793 * u2);
      if (axis == 0)
        x = z0 * L.sigma + x;
      else
        y = z0 * L.sigma + y;
    }
  }
  const double t0 = L.time_offset * 1e-3;
  t = t0;
  switch (L.temporal) {
  case 1: {
    const double u1 = (double)uniform<R>(g, rp);
    const double u2 = (double)uniform<R>(g, rp);
    const double z0 = sqrt(-2.0 * log(u1)) * cos(2.0 * 3.141592653589793 * u2);
    t = z0 * (L.pulse_duration * (1.0 / (2.0 * sqrt(2.0 * log(2.0)))) * 1e-3) + t0;
    break;
  }
  case 2: t = t0 + ((double)uniform<R>(g, rp) - 0.5) * L.pulse_duration * 1e-3; break;
  case 3: t = t0 - log((double)uniform<R>(g, rp)) * L.pulse_duration * 1e-3; break;
  case 4: t = (L.repetition_rate <= 0.0) ? t0 : t0 + (double)uniform<R>(g, rp) * (1e9 / L.repetition_rate); break;
  case 5: t = (L.pulse_duration <= 0.0) ? t0 : t0 + (double)uniform<R>(g, rp) * L.pulse_duration * 1e-3; break;
  default: break;
  }
}

// Emission time of photon `index`, re-derived from its stream (counter-based, so
// draws 0.. can be regenerated at any time) instead of carried in registers.
template <typename R>
__device__ __noinline__ double emission_time(const Laser &L, RunParams rp, unsigned long long index)
{
  if (L.temporal == 0)
    return L.time_offset * 1e-3;
  uint32_t words[kRing];                  // a private ring (local memory; rare path)
  RngT<1> g;
  g.ring = words;
  rng_reset(g, index);
  double x, y, t;
  source_sample<R>(L, g, rp, x, y, t);
  return t;
}

template <typename R>
__device__ __forceinline__ double launch_time(const Scene &sc, const RunParams &rp, const Photon<R> &ph)
{
  return emission_time<R>(sc.laser, rp, ph.index());
}

// ---------------------------------------------------------------- hit snapshot
// What a sensor's process_hit reads from the photon at a plane crossing.
template <typename R> struct HitData {
  uint32_t p_lo, p_hi, events, first_med, last_med;
  double w, opath;             // weight, geometric path length at the hit point
  double pen;                  // penetration depth (StatisticsSensor)
  R hx, hy, hz;                // hit point
  R P[9];                      // P_local rows m, n, s
  Cx<R> Em, En;
  R r1[3], rn[3];              // CBS: first and newest scatter positions
  R P1[9], Pn1[9];             // CBS: frame after the first scatter, before the newest
  Cx<R> T[4];                  // CBS: interior Jones product
};

// ---------------------------------------------------------------- CBS reverse path
// reverse_field (src/detector.cpp:1080-1173): stages A (scatter at r_n), B
// (interior by reciprocity, Q T^T Q) and C (scatter at r_1), normalised once.
template <typename R>
__device__ void reverse_field(const Scene &sc, const HitData<R> &h, Cx<R> &Om, Cx<R> &On)
{
  const Laser &L = sc.laser;
  const V3<R> m0 = v3<R>(R(L.m[0]), R(L.m[1]), R(L.m[2]));
  const V3<R> n0 = v3<R>(R(L.n[0]), R(L.n[1]), R(L.n[2]));
  const V3<R> s0 = v3<R>(R(L.dir[0]), R(L.dir[1]), R(L.dir[2]));
  const Cx<R> E0m = {R(L.E[0]), R(L.E[1])}, E0n = {R(L.E[2]), R(L.E[3])};
  // Stage A: s0 -> -s_{n-1} at r_n, species of the last vertex
  const V3<R> mnm1 = row(h.Pn1, 0), nnm1 = row(h.Pn1, 1), snm1 = row(h.Pn1, 2);
  const V3<R> s_out_a = vscale(snm1, R(-1));
  Cx<R> Sa2, Sa1;
  amplitudes<R>(sc.media[h.last_med], unit_angle(s0, s_out_a), Sa2, Sa1);
  const V3<R> np_ = safe_unit(vcross_unit(s0, s_out_a), n0);
  const V3<R> mp_in = safe_unit(vcross_unit(np_, s0), m0);
  const V3<R> mp_out = safe_unit(vcross_unit(np_, s_out_a), mnm1);
  R r00 = vdot(mp_in, m0), r01 = vdot(mp_in, n0), r10 = vdot(np_, m0), r11 = vdot(np_, n0);
  Cx<R> Em = cadd(cmul(cscale(Sa2, r00), E0m), cmul(cscale(Sa2, r01), E0n));
  Cx<R> En = cadd(cmul(cscale(Sa1, r10), E0m), cmul(cscale(Sa1, r11), E0n));
  const V3<R> nn1 = vscale(nnm1, R(-1));
  r00 = vdot(mnm1, mp_out); r01 = vdot(mnm1, np_); r10 = vdot(nn1, mp_out); r11 = vdot(nn1, np_);
  Cx<R> tm = cadd(cscale(Em, r00), cscale(En, r01));
  Cx<R> tn = cadd(cscale(Em, r10), cscale(En, r11));
  // Stage B: E <- Q T^T Q E, Q = diag(1, -1)
  tn = {-tn.re, -tn.im};
  Em = cadd(cmul(h.T[0], tm), cmul(h.T[2], tn));
  En = cadd(cmul(h.T[1], tm), cmul(h.T[3], tn));
  En = {-En.re, -En.im};
  // Stage C: -s_1 -> s_n at r_1, species of the first vertex
  const V3<R> m1 = row(h.P1, 0), n1 = row(h.P1, 1), s1 = row(h.P1, 2);
  const V3<R> mn = row(h.P, 0), nn = row(h.P, 1), sn = row(h.P, 2);
  const V3<R> s_in_c = vscale(s1, R(-1));
  const V3<R> n1m = vscale(n1, R(-1));
  Cx<R> Sc2, Sc1;
  amplitudes<R>(sc.media[h.first_med], unit_angle(s_in_c, sn), Sc2, Sc1);
  const V3<R> npp = safe_unit(vcross_unit(s_in_c, sn), n1m);
  const V3<R> mpp_in = safe_unit(vcross_unit(npp, s_in_c), m1);
  const V3<R> mpp_out = safe_unit(vcross_unit(npp, sn), mn);
  r00 = vdot(mpp_in, m1); r01 = vdot(mpp_in, n1m); r10 = vdot(npp, m1); r11 = vdot(npp, n1m);
  const Cx<R> Fm = cadd(cmul(cscale(Sc2, r00), Em), cmul(cscale(Sc2, r01), En));
  const Cx<R> Fn = cadd(cmul(cscale(Sc1, r10), Em), cmul(cscale(Sc1, r11), En));
  r00 = vdot(mn, mpp_out); r01 = vdot(mn, npp); r10 = vdot(nn, mpp_out); r11 = vdot(nn, npp);
  Cx<R> gm = cadd(cscale(Fm, r00), cscale(Fn, r01));
  Cx<R> gn = cadd(cscale(Fm, r10), cscale(Fn, r11));
  const R nrm = m_sqrt(cnorm(gm) + cnorm(gn));
  if (nrm > tiny<R>()) {
    gm = {gm.re / nrm, gm.im / nrm};
    gn = {gn.re / nrm, gn.im / nrm};
  } else {
    gm = {R(0), R(0)};
    gn = {R(0), R(0)};
  }
  Om = gm;
  On = gn;
}

// ------------------------------------------------------------------- tallies
// Tally modes of the hit-queue tally kernel (lmc_tally_mode less one): every add a
// global atomic; lanes of a warp adding into one cell combined first; block-private
// shared-memory grids for the sensors the run privatises.
constexpr int kTallyGlobal = 0, kTallyWarp = 1, kTallyShared = 2;

// The four Stokes values of one cell: planes base, base + stride, ... at `off`.
// kTallyWarp: the lanes of the warp that reach this call together group by cell
// (__match_any_sync on the address); the lowest lane of each group pulls its peers'
// values one lane at a time by shuffles and issues the group's four atomics.  When no
// two lanes share a cell (the common case) that costs one match and one vote.
template <int kT = kTallyGlobal>
__device__ __forceinline__ void add4(double *base, unsigned long long stride, unsigned long long off,
                                     double a, double b, double c, double d)
{
  double *const p = base + off;
  if (kT == kTallyWarp) {
    const unsigned act = __activemask();
    const unsigned lane = threadIdx.x & 31u;
    const unsigned peers = __match_any_sync(act, (unsigned long long)p);
    const bool lead = (unsigned)(__ffs(peers) - 1) == lane;
    if (__any_sync(act, peers != (1u << lane))) {
      double sa = a, sb = b, sc = c, sd = d;
      unsigned pend = lead ? (peers & ~(1u << lane)) : 0u;
      while (__any_sync(act, pend != 0u)) {
        const int src = pend ? __ffs(pend) - 1 : (int)lane;
        const double ta = __shfl_sync(act, a, src), tb = __shfl_sync(act, b, src);
        const double tc = __shfl_sync(act, c, src), td = __shfl_sync(act, d, src);
        if (pend) {
          sa += ta; sb += tb; sc += tc; sd += td;
          pend &= pend - 1u;
        }
      }
      a = sa; b = sb; c = sc; d = sd;
    }
    if (!lead)
      return;
  }
  atomicAdd(p, a);
  atomicAdd(p + stride, b);
  atomicAdd(p + 2 * stride, c);
  atomicAdd(p + 3 * stride, d);
}

// Where sensor si's adds go: its block-private copy in shared memory (kTallyShared,
// when the run privatised it; the generic-address atomics then resolve to shared
// memory), else the tally buffer.
template <int kT>
__device__ __forceinline__ double *tally_base(const RunParams &rp, const Sensor &s, int si, double *priv)
{
  if (kT == kTallyShared && rp.tally_smem[si] >= 0)
    return priv + rp.tally_smem[si];
  return rp.tallies + s.tally_off;
}

__device__ __forceinline__ int time_bin(const Sensor &s, double arrival)
{                                                          // src/detector.cpp:1182-1190
  if (s.dt <= 0)
    return 0;
  if (arrival < 0 || arrival >= s.len_t)
    return -1;
  const int idx = (int)(arrival / s.dt) + 1;
  return (idx < s.N_t) ? idx : -1;
}

template <typename R>
__device__ __forceinline__ double hit_launch_time(const Scene &sc, const RunParams &rp, const HitData<R> &h)
{
  return emission_time<R>(sc.laser, rp, ((unsigned long long)h.p_hi << 32) | h.p_lo);
}

// The likelihood-ratio output layout a hit contributes to: the run's (one scene), or
// its scene's block of a sweep.
struct AdjView {
  double *out;                 // row 0 of the block; row 1 + k at out + (1 + k) n_out
  unsigned long long n_out;
  int K, radial_sensor, radial_bins;
  double radial_max;
  const unsigned long long *cbs_off;
};

template <bool kSweep>
__device__ __forceinline__ AdjView adj_view(const RunParams &rp, unsigned scene)
{
  if (kSweep) {
    const AdjScene &a = rp.adj_scenes[scene];
    return {rp.adj_out + a.out_off, a.n_out, a.K, a.radial_sensor, a.radial_bins, a.radial_max,
            a.cbs_off};
  }
  return {rp.adj_out, rp.adj_n_out, rp.adj_K, rp.adj_radial_sensor, rp.adj_radial_bins,
          rp.adj_radial_max, rp.adj_cbs_off};
}

// Likelihood-ratio outputs of one hit contribution v: row 0 += v, row 1 + k +=
// v * score_k.  Global atomics (FarFieldCBS bins; the radial outputs of a sweep), or
// the block's shared-memory copy of the radial outputs (rows of radial_bins + 1).
template <typename R>
__device__ __forceinline__ void adj_add_global(const AdjView &A, unsigned long long idx, double v,
                                               const R *hs)
{
  atomicAdd(A.out + idx, v);
  for (int k = 0; k < A.K; ++k)
    atomicAdd(A.out + (unsigned long long)(1 + k) * A.n_out + idx, v * (double)hs[k]);
}

template <typename R>
__device__ __forceinline__ void adj_add_radial(const AdjView &A, double *s_rad, int idx, double v,
                                               const R *hs)
{
  if (!s_rad) {
    adj_add_global<R>(A, (unsigned long long)idx, v, hs);
    return;
  }
  const int row = A.radial_bins + 1;
  atomicAdd(s_rad + idx, v);
  for (int k = 0; k < A.K; ++k)
    atomicAdd(s_rad + (1 + k) * row + idx, v * (double)hs[k]);
}

// FarFieldCBSSensor::process_hit (src/detector.cpp:1231-1310) and the far-field
// fluence sensor (same binning, reverse field zero).  exp(i k L) multiplies E_f
// and E_r alike and cancels in every Stokes parameter, so it is not formed.
template <typename R, bool kAdj, int kT = kTallyGlobal>
__device__ bool hit_farfield(const Scene &sc, const RunParams &rp, const Sensor &s,
                             const HitData<R> &h, lmc_record *rec, int si, const R *hs, const AdjView *A,
                             double *priv = nullptr)
{
  const double t_launch = (s.dt > 0) ? hit_launch_time<R>(sc, rp, h) : 0.0;
  const int t_idx = time_bin(s, t_launch + h.opath);
  if (t_idx < 0)
    return false;
  const R sx = h.P[6], sy = h.P[7], sz = h.P[8];
  const R theta = exit_theta(sx, sy, sz);
  R phi = m_atan2(sy, sx);
  if (phi < R(0))
    phi += R(6.283185307179586);
  const int it = (int)(theta / R(s.dtheta));
  const int jp = (int)(phi / R(s.dphi));
  if (it < 0 || it >= s.N_theta || jp < 0 || jp >= s.N_phi)
    return false;
  const R w_sqrt = R(sqrt(h.w));
  const Cx<R> Em = cscale(h.Em, w_sqrt), En = cscale(h.En, w_sqrt);
  // project_to_lab (src/detector.cpp:1048-1053)
  const Cx<R> Efx = cadd(cscale(Em, h.P[0]), cscale(En, h.P[3]));
  const Cx<R> Efy = cadd(cscale(Em, h.P[1]), cscale(En, h.P[4]));
  const unsigned long long cell = ((unsigned long long)it) * s.N_phi + jp;
  const unsigned long long tstride = (unsigned long long)s.N_theta * s.N_phi;
  double *base = tally_base<kT>(rp, s, si, priv);
  const unsigned long long P = s.plane_stride;
  if (!in_bounds(kBoundFarfield, (unsigned long long)t_idx * tstride + cell < P))
    return false;
  if (s.kind == LMC_SENSOR_FARFIELD_FLUENCE) {
    const double q0 = (double)(cnorm(Efx) + cnorm(Efy)), q1 = (double)(cnorm(Efx) - cnorm(Efy));
    const Cx<R> xy = cmul(Efx, Cx<R>{Efy.re, -Efy.im});
    const double q2 = 2.0 * (double)xy.re, q3 = 2.0 * (double)xy.im;
    add4<kT>(base, P, cell, q0, q1, q2, q3);
    if (t_idx >= 1)
      add4<kT>(base, P, t_idx * tstride + cell, q0, q1, q2, q3);
    return true;
  }
  Cx<R> Erx = {R(0), R(0)}, Ery = {R(0), R(0)};
  if (h.events >= 2) {
    Cx<R> Rm, Rn;
    reverse_field<R>(sc, h, Rm, Rn);
    if (rec) {                     // photon.polarization_reverse, kept for the replay check
      rec->Er[0] = Rm.re; rec->Er[1] = Rm.im; rec->Er[2] = Rn.re; rec->Er[3] = Rn.im;
    }
    // CBS geometric phase exp(i k (s_out + s_in).(r_n - r_1)) in binary64, or all in
    // binary32 when the run asks for it (precision study)
    const Laser &L = sc.laser;
    double sp, cp;
    if (rp.cbs_phase_f32) {
      const float kf = (float)L.k;
      const float qx = ((float)sx + (float)L.dir[0]) * kf, qy = ((float)sy + (float)L.dir[1]) * kf,
                  qz = ((float)sz + (float)L.dir[2]) * kf;
      const float arg = qx * ((float)h.rn[0] - (float)h.r1[0]) + qy * ((float)h.rn[1] - (float)h.r1[1]) +
                        qz * ((float)h.rn[2] - (float)h.r1[2]);
      float spf, cpf;
      sincosf(arg, &spf, &cpf);
      sp = spf;
      cp = cpf;
    } else {
      const double qx = ((double)sx + L.dir[0]) * L.k, qy = ((double)sy + L.dir[1]) * L.k,
                   qz = ((double)sz + L.dir[2]) * L.k;
      const double arg = qx * ((double)h.rn[0] - (double)h.r1[0]) +
                         qy * ((double)h.rn[1] - (double)h.r1[1]) +
                         qz * ((double)h.rn[2] - (double)h.r1[2]);
      sincos(arg, &sp, &cp);
    }
    const Cx<R> pp = {R(cp), R(sp)};
    const Cx<R> Rm2 = cmul(cscale(Rm, w_sqrt), pp), Rn2 = cmul(cscale(Rn, w_sqrt), pp);
    Erx = cadd(cscale(Rm2, h.P[0]), cscale(Rn2, h.P[3]));
    Ery = cadd(cscale(Rm2, h.P[1]), cscale(Rn2, h.P[4]));
  }
  // accumulate_stokes (src/detector.cpp:1194-1226)
  const Cx<R> Ex = cadd(Efx, Erx), Ey = cadd(Efy, Ery);
  const Cx<R> c_xy = cmul(Ex, Cx<R>{Ey.re, -Ey.im});
  const Cx<R> f_xy = cmul(Efx, Cx<R>{Efy.re, -Efy.im});
  const Cx<R> r_xy = cmul(Erx, Cx<R>{Ery.re, -Ery.im});
  const double c0 = (double)(cnorm(Ex) + cnorm(Ey)), c1 = (double)(cnorm(Ex) - cnorm(Ey));
  const double c2 = 2.0 * (double)c_xy.re, c3 = 2.0 * (double)c_xy.im;
  const double i0 = (double)(cnorm(Efx) + cnorm(Efy) + cnorm(Erx) + cnorm(Ery));
  const double i1 = (double)(cnorm(Efx) - cnorm(Efy) + cnorm(Erx) - cnorm(Ery));
  const double i2 = 2.0 * ((double)f_xy.re + (double)r_xy.re);
  const double i3 = 2.0 * ((double)f_xy.im + (double)r_xy.im);
  add4<kT>(base, P, cell, c0, c1, c2, c3);
  add4<kT>(base + 4 * P, P, cell, i0, i1, i2, i3);
  if (t_idx >= 1) {
    add4<kT>(base, P, t_idx * tstride + cell, c0, c1, c2, c3);
    add4<kT>(base + 4 * P, P, t_idx * tstride + cell, i0, i1, i2, i3);
  }
  if (kAdj && s.kind == LMC_SENSOR_FARFIELD_CBS) {     // S0 coherent, S0 incoherent
    const unsigned long long o = A->cbs_off[si];
    adj_add_global<R>(*A, o + cell, c0, hs);
    adj_add_global<R>(*A, o + P + cell, i0, hs);
    if (t_idx >= 1) {
      adj_add_global<R>(*A, o + t_idx * tstride + cell, c0, hs);
      adj_add_global<R>(*A, o + P + t_idx * tstride + cell, i0, hs);
    }
  }
  return true;
}

// PlanarFluenceSensor::process_hit (src/detector.cpp:780-841): lab-frame Stokes
// with E_x negated; exp(i k L) cancels and is not formed.
template <typename R, bool kAdj, int kT = kTallyGlobal>
__device__ bool hit_fluence(const Scene &sc, const RunParams &rp, const Sensor &s, const HitData<R> &h,
                            int si, const R *hs, double *s_rad, const AdjView *A, double *priv = nullptr)
{
  int t_idx = -1;
  if (s.dt > 0) {
    const double arrival = hit_launch_time<R>(sc, rp, h) + h.opath;
    if (arrival < 0 || arrival >= s.len_t)
      return false;
    t_idx = (int)(arrival / s.dt) + 1;
    if (t_idx >= s.N_t)
      return false;
  }
  const int xi = (int)(((double)h.hx + 0.5 * s.len_x) / s.dx);
  const int yi = (int)(((double)h.hy + 0.5 * s.len_y) / s.dy);
  if (xi < 0 || xi >= s.N_x || yi < 0 || yi >= s.N_y)
    return false;
  const R w_sqrt = R(sqrt(h.w));
  const Cx<R> Em = cscale(h.Em, w_sqrt), En = cscale(h.En, w_sqrt);
  const Cx<R> Ex = cscale(cadd(cscale(Em, h.P[0]), cscale(En, h.P[3])), R(-1));
  const Cx<R> Ey = cadd(cscale(Em, h.P[1]), cscale(En, h.P[4]));
  const Cx<R> xy = cmul(Ex, Cx<R>{Ey.re, -Ey.im});
  const double q0 = (double)(cnorm(Ex) + cnorm(Ey)), q1 = (double)(cnorm(Ex) - cnorm(Ey));
  const double q2 = 2.0 * (double)xy.re, q3 = 2.0 * (double)xy.im;
  double *base = tally_base<kT>(rp, s, si, priv);
  const unsigned long long cell = (unsigned long long)xi * s.N_y + yi;
  const unsigned long long tstride = (unsigned long long)s.N_x * s.N_y;
  if (!in_bounds(kBoundFluence, (unsigned long long)(t_idx > 0 ? t_idx : 0) * tstride + cell < s.plane_stride))
    return false;
  if (s.dt > 0)
    add4<kT>(base, s.plane_stride, t_idx * tstride + cell, q0, q1, q2, q3);
  add4<kT>(base, s.plane_stride, cell, q0, q1, q2, q3);
  if (kAdj && si == A->radial_sensor) {                // total S0 and its radial profile
    adj_add_radial<R>(*A, s_rad, 0, q0, hs);
    const double r = sqrt((double)h.hx * (double)h.hx + (double)h.hy * (double)h.hy);
    if (r < A->radial_max) {
      const int ir = (int)(r / (A->radial_max / A->radial_bins));
      if (ir >= 0 && ir < A->radial_bins)
        adj_add_radial<R>(*A, s_rad, 1 + ir, q0, hs);
    }
  }
  return true;
}

// PlanarFieldSensor::process_hit (src/detector.cpp:546-568): complex field with
// the propagation phase exp(i k L), L = n * (path length at the hit).
template <typename R>
__device__ bool hit_field(const Scene &sc, const RunParams &rp, const Sensor &s, const HitData<R> &h)
{
  const int xi = (int)(((double)h.hx + 0.5 * s.len_x) / s.dx);
  const int yi = (int)(((double)h.hy + 0.5 * s.len_y) / s.dy);
  if (xi < 0 || xi >= s.N_x || yi < 0 || yi >= s.N_y)
    return false;
  double pi, pr;
  sincos(sc.laser.k * (sc.n_step * h.opath), &pi, &pr);
  const double w_sqrt = sqrt(h.w);
  const double P0 = h.P[0], P1 = h.P[1], P3 = h.P[3], P4 = h.P[4];
  const double exr = (double)h.Em.re * P0 + (double)h.En.re * P3;
  const double exi = (double)h.Em.im * P0 + (double)h.En.im * P3;
  const double eyr = (double)h.Em.re * P1 + (double)h.En.re * P4;
  const double eyi = (double)h.Em.im * P1 + (double)h.En.im * P4;
  double *base = rp.tallies + s.tally_off;
  const unsigned long long off = ((unsigned long long)xi * s.N_y + yi) * 2;
  if (!in_bounds(kBoundField, off + 1 < s.plane_stride))
    return false;
  atomicAdd(base + off, (exr * pr - exi * pi) * w_sqrt);
  atomicAdd(base + off + 1, (exr * pi + exi * pr) * w_sqrt);
  atomicAdd(base + s.plane_stride + off, (eyr * pr - eyi * pi) * w_sqrt);
  atomicAdd(base + s.plane_stride + off + 1, (eyr * pi + eyi * pr) * w_sqrt);
  return true;
}

// StatisticsSensor::process_hit (src/detector.cpp:1720-1800): one count in every
// histogram the hit falls in, in slice 0 and in the arrival-time window of the four
// time-resolved ones.  Bins past a histogram's end are skipped.  Always counted.
// Out of line with scalar arguments (arrival time, events, exit direction s,
// penetration depth, weight), so that the callers' hit state stays in registers.
__device__ __noinline__ void hit_statistics(const Sensor &s, double *tallies, double arrival,
                                            uint32_t events, double sx, double sy, double sz,
                                            double pen, double w)
{
  const StatHist &q = *s.stat;
  int t_idx = -1;
  if (s.N_t > 1 && s.dt > 0.0 && arrival >= 0.0 && arrival < s.len_t) {
    t_idx = (int)(arrival / s.dt) + 1;
    if (t_idx >= s.N_t)
      t_idx = -1;
  }
  double *base = tallies + s.tally_off;
  auto deposit = [&](unsigned long long off, int nb, int idx) {
    if (idx >= 0 && idx < nb) {
      atomicAdd(base + off + idx, 1.0);
      if (t_idx >= 1)
        atomicAdd(base + off + (unsigned long long)t_idx * nb + idx, 1.0);
    }
  };
  if (q.set & LMC_STAT_EVENTS) {
    if ((int)events >= 0 && (int)events < q.n_events)
      deposit(q.off[0], q.n_events, (int)events);
  }
  if (q.set & LMC_STAT_THETA) {
    const double theta = acos(-sz);
    if (theta >= q.theta_min && theta < q.theta_max)
      deposit(q.off[1], q.n_theta, (int)((theta - q.theta_min) / q.dtheta));
  }
  if (q.set & LMC_STAT_PHI) {
    double phi = atan2(sy, sx);
    if (phi < 0)
      phi += 2.0 * 3.141592653589793;
    if (phi >= q.phi_min && phi < q.phi_max)
      deposit(q.off[2], q.n_phi, (int)((phi - q.phi_min) / q.dphi));
  }
  if (q.set & LMC_STAT_DEPTH) {
    if (pen >= 0 && pen < q.depth_max)
      deposit(q.off[3], q.n_depth, (int)(pen / q.ddepth));
  }
  if (q.set & LMC_STAT_TIME) {
    const double fi = arrival / q.dtime;
    if (fi >= 1.0 && fi < (double)q.n_time)
      atomicAdd(base + q.off[4] + (unsigned long long)fi, 1.0);
  }
  if (q.set & LMC_STAT_WEIGHT) {
    if (w >= 0 && w < q.weight_max) {
      const int idx = (int)(w / q.dweight);
      if (idx < q.n_weight)
        atomicAdd(base + q.off[5] + idx, 1.0);
    }
  }
}

// process_hit of every sensor in `mask` (all on the plane of this hit), in
// insertion order, as SensorsGroup::record_hit calls them (src/detector.cpp:244-265).
// kT: the tally kernel's mode (kTallyShared: priv is the block's private grid area).
template <typename R, bool kAdj, int kT = kTallyGlobal>
__device__ void process_hits(const Scene &sc, const RunParams &rp, const HitData<R> &h,
                             unsigned mask, unsigned long long *hits, const R *hs, double *s_rad,
                             const AdjView *A, double *priv = nullptr)
{
  lmc_record *rec = rp.records ? rp.records + ((((unsigned long long)h.p_hi << 32) | h.p_lo) -
                                               rp.photon_begin)
                               : nullptr;
  for (int si = 0; si < sc.n_sensors; ++si) {
    if (!(mask & (1u << si)))
      continue;
    const Sensor &s = sc.sensors[si];
    bool counted;
    if (s.kind == LMC_SENSOR_PLANAR_FLUENCE)
      counted = hit_fluence<R, kAdj, kT>(sc, rp, s, h, si, hs, s_rad, A, priv);
    else if (s.kind == LMC_SENSOR_PLANAR_FIELD)
      counted = hit_field<R>(sc, rp, s, h);
    else if (s.kind == LMC_SENSOR_STATISTICS) {
      const double arrival = (s.dt > 0 || (s.stat->set & LMC_STAT_TIME))
                                 ? hit_launch_time<R>(sc, rp, h) + h.opath : 0.0;
      double d[3];
      exit_dir(h.P[6], h.P[7], h.P[8], d);
      hit_statistics(s, rp.tallies, arrival, h.events, d[0], d[1], d[2], h.pen, h.w);
      counted = true;
    }
    else
      counted = hit_farfield<R, kAdj, kT>(sc, rp, s, h, rec, si, hs, A, priv);
    if (counted && rec) {
      rec->hit[0] = h.hx;
      rec->hit[1] = h.hy;
      rec->hit[2] = h.hz;
      atomicAdd(&rec->n_hits, 1);
    }
    // Sensor::hits: the lanes here that count into the same counter (a block's shared
    // counters, or a sweep scene's) add their number in one atomic, from their lowest
    // lane; one atomic per lane serialised the warp on a few shared addresses
    const unsigned act = __activemask();
    unsigned long long *const cp = hits + si;
    const unsigned grp = __match_any_sync(act, (unsigned long long)cp);
    const unsigned cnt = __ballot_sync(act, counted) & grp;
    if ((threadIdx.x & 31u) == (unsigned)(__ffs(grp) - 1) && cnt)
      atomicAdd(cp, (unsigned long long)__popc(cnt));
  }
}

// ------------------------------------------------ last-flight CBS estimator
// FarFieldCBSSensor::process_estimation (src/detector.cpp:1315-1566).  At every
// scattering vertex, before the scatter is sampled, the photon is forced toward the
// centre of every angular bin of an estimator-mode FarFieldCBS grid.  The bin gets the
// weight w mu_s / mu_t x transmittance to the plane x p(Omega) dOmega, with
// p = F / (pi I_norm), and the forward field.  From the second vertex on it also gets
// the reverse (CBS) field with its geometric phase.
__device__ __forceinline__ V3<double> drow(const double *P, int r)
{
  return v3<double>(P[3 * r], P[3 * r + 1], P[3 * r + 2]);
}

template <typename T> __device__ __forceinline__ V3<T> trow(const T *P, int r)
{
  return v3<T>(P[3 * r], P[3 * r + 1], P[3 * r + 2]);
}

// Stages A + B of the reverse path with P_{n-1} = the current frame
// (src/detector.cpp:1079-1118).
template <typename T>
__device__ __forceinline__ void est_prefix(const Scene &sc, const T *Pnm1, const Cx<T> *Tm,
                                           int med_n, Cx<T> &Om, Cx<T> &On)
{
  const Laser &L = sc.laser;
  const V3<T> m0 = v3<T>(T(L.m[0]), T(L.m[1]), T(L.m[2]));
  const V3<T> n0 = v3<T>(T(L.n[0]), T(L.n[1]), T(L.n[2]));
  const V3<T> s0 = v3<T>(T(L.dir[0]), T(L.dir[1]), T(L.dir[2]));
  const Cx<T> E0m = {T(L.E[0]), T(L.E[1])}, E0n = {T(L.E[2]), T(L.E[3])};
  const V3<T> mnm1 = trow<T>(Pnm1, 0), nnm1 = trow<T>(Pnm1, 1), snm1 = trow<T>(Pnm1, 2);
  const V3<T> s_out_a = vscale(snm1, T(-1));
  Cx<T> Sa2, Sa1;
  amplitudes<T>(sc.media[med_n], unit_angle(s0, s_out_a), Sa2, Sa1);
  const V3<T> np_ = safe_unit(vcross_unit(s0, s_out_a), n0);
  const V3<T> mp_in = safe_unit(vcross_unit(np_, s0), m0);
  const V3<T> mp_out = safe_unit(vcross_unit(np_, s_out_a), mnm1);
  T r00 = vdot(mp_in, m0), r01 = vdot(mp_in, n0), r10 = vdot(np_, m0), r11 = vdot(np_, n0);
  Cx<T> Em = cadd(cmul(cscale(Sa2, r00), E0m), cmul(cscale(Sa2, r01), E0n));
  Cx<T> En = cadd(cmul(cscale(Sa1, r10), E0m), cmul(cscale(Sa1, r11), E0n));
  const V3<T> nn1 = vscale(nnm1, T(-1));
  r00 = vdot(mnm1, mp_out); r01 = vdot(mnm1, np_); r10 = vdot(nn1, mp_out); r11 = vdot(nn1, np_);
  Cx<T> tm = cadd(cscale(Em, r00), cscale(En, r01));
  Cx<T> tn = cadd(cscale(Em, r10), cscale(En, r11));
  tn = {-tn.re, -tn.im};
  Em = cadd(cmul(Tm[0], tm), cmul(Tm[2], tn));
  En = cadd(cmul(Tm[1], tm), cmul(Tm[3], tn));
  Om = Em;
  On = {-En.re, -En.im};
}

// Stage C and the normalisation (src/detector.cpp:1122-1161).
template <typename T>
__device__ __forceinline__ void est_suffix(const Scene &sc, const T *P1, const T *Pn, int med_1,
                                           Cx<T> Em, Cx<T> En, Cx<T> &Om, Cx<T> &On)
{
  const V3<T> m1 = trow<T>(P1, 0), n1 = trow<T>(P1, 1), s1 = trow<T>(P1, 2);
  const V3<T> mn = trow<T>(Pn, 0), nn = trow<T>(Pn, 1), sn = trow<T>(Pn, 2);
  const V3<T> s_in_c = vscale(s1, T(-1));
  const V3<T> n1m = vscale(n1, T(-1));
  Cx<T> Sc2, Sc1;
  amplitudes<T>(sc.media[med_1], unit_angle(s_in_c, sn), Sc2, Sc1);
  const V3<T> npp = safe_unit(vcross_unit(s_in_c, sn), n1m);
  const V3<T> mpp_in = safe_unit(vcross_unit(npp, s_in_c), m1);
  const V3<T> mpp_out = safe_unit(vcross_unit(npp, sn), mn);
  T r00 = vdot(mpp_in, m1), r01 = vdot(mpp_in, n1m), r10 = vdot(npp, m1), r11 = vdot(npp, n1m);
  const Cx<T> Fm = cadd(cmul(cscale(Sc2, r00), Em), cmul(cscale(Sc2, r01), En));
  const Cx<T> Fn = cadd(cmul(cscale(Sc1, r10), Em), cmul(cscale(Sc1, r11), En));
  r00 = vdot(mn, mpp_out); r01 = vdot(mn, npp); r10 = vdot(nn, mpp_out); r11 = vdot(nn, npp);
  Cx<T> gm = cadd(cscale(Fm, r00), cscale(Fn, r01));
  Cx<T> gn = cadd(cscale(Fm, r10), cscale(Fn, r11));
  const T nrm = sqrt(cnorm(gm) + cnorm(gn));
  if (nrm > tiny<T>()) {
    gm = {gm.re / nrm, gm.im / nrm};
    gn = {gn.re / nrm, gn.im / nrm};
  } else {
    gm = {T(0), T(0)};
    gn = {T(0), T(0)};
  }
  Om = gm;
  On = gn;
}

// Optical depth of a straight ray to the detector plane, layer by layer
// (src/detector.cpp:52-102).
__device__ __forceinline__ double est_optical_depth(const Scene &sc, const double *start, V3<double> dir,
                                                    double L_total)
{
  double tau = 0.0, traveled = 0.0;
  double px = start[0], py = start[1], pz = start[2];
  int layer = layer_index_at<double>(sc, pz);
  if (layer >= sc.n_layers)
    return 0.0;
  if (sc.n_layers == 1)
    return sc.layers[layer].mu_t * L_total;
  const double dz = dir.z;
  for (int guard = 0; guard <= 2 * LMC_MAX_LAYERS && traveled < L_total - 1e-15; ++guard) {
    const double remaining = L_total - traveled;
    const double mu = sc.layers[layer].mu_t;
    double seg = remaining;
    if (fabs(dz) > 1e-15) {
      double zi;
      if (find_next_interface<double>(sc, pz, pz + dz * remaining, zi)) {
        const double sd = (zi - pz) / dz;
        if (sd > 1e-15 && sd < remaining)
          seg = sd;
      }
    }
    tau += mu * seg;
    px += dir.x * seg;
    py += dir.y * seg;
    pz += dir.z * seg;
    traveled += seg;
    if (seg >= remaining - 1e-15)
      break;
    const int next = layer_index_at<double>(sc, pz + ((dz > 0) ? 1e-12 : -1e-12));
    if (next >= sc.n_layers)
      break;
    layer = next;
  }
  return tau;
}

// ------------------------------------------------ warp-cooperative estimation
// The 32 lanes of a warp estimate together.  Every lane whose photon is at a vertex
// prepares it (filters, weight, the reverse-path prefix, launch time); the warp then
// takes the prepared vertices one at a time, broadcast by shuffles, and lane j
// evaluates bins j, j + 32, ... of the grid.  A vertex so deep that the
// transmittance to the plane is below the reference's cut (1e-20) for every bin is
// skipped by the whole warp instead of by each bin.  The 32 lanes of one step write
// 32 different cells, so a warp can accumulate into a private copy of the grid
// with plain adds.

// Where a sensor's estimate accumulates: the warp's private copy of the grid in
// shared memory (plain adds), the block's shared copy (shared atomics: several warps
// write it), or the tallies (global atomics).
struct EstTarget {
  double *base;
  bool atomic;
  __device__ __forceinline__ void add(unsigned long long off, double v) const
  {
    if (atomic)
      atomicAdd(base + off, v);
    else
      base[off] += v;
  }
  __device__ __forceinline__ void add4(unsigned long long stride, unsigned long long off, double a,
                                       double b, double c, double d) const
  {
    add(off, a);
    add(stride + off, b);
    add(2 * stride + off, c);
    add(3 * stride + off, d);
  }
};

__device__ __forceinline__ EstTarget est_target(const RunParams &rp, const Sensor &s, int si, double *s_est)
{
  if (rp.est_smem[si] < 0)
    return {rp.tallies + s.tally_off, true};
  if (rp.est_per_warp)
    return {s_est + (threadIdx.x >> 5) * rp.est_warp_doubles + rp.est_smem[si], false};
  return {s_est + rp.est_smem[si], true};
}

// A vertex as the estimate reads it, in the estimate's precision T (binary64 for
// binary64 transport, binary32 for binary32 transport, whose positions are binary32
// already).  Small, because every lane holds its own vertex and the one broadcast:
// r_1 and the frame after the first scatter stay in the source lane's Side column in
// shared memory, where the bin reads them.
template <typename T> struct EstV {
  T P[9];                       // frame at the vertex
  Cx<T> Em, En;                 // Jones vector
  Cx<T> pre_m, pre_n;           // reverse path through stages A + B (from the 2nd vertex)
  T pos[3];                     // vertex
  T wgt;                        // binary64: w mu_s / mu_t; binary32: that / (pi I_norm)
  double opath, t_launch;       // broadcast only for a time-resolved grid
  int ids;                      // medium | first medium << 8 | layer << 16 | multi << 24
  __device__ __forceinline__ int med() const { return ids & 0xff; }
  __device__ __forceinline__ int first_med() const { return (ids >> 8) & 0xff; }
  __device__ __forceinline__ int layer() const { return (ids >> 16) & 0xff; }
  __device__ __forceinline__ bool multi() const { return (ids >> 24) & 1; }
};

// Every lane takes the vertex of lane src (its own source; lanes may differ): the
// fields the bin loop reads, opath and the launch time only for a time-resolved grid.
template <typename T> __device__ __forceinline__ void est_fetch(EstV<T> &v, int src, bool timed)
{
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    v.P[j] = __shfl_sync(kFull, v.P[j], src);
  }
  v.Em.re = __shfl_sync(kFull, v.Em.re, src);
  v.Em.im = __shfl_sync(kFull, v.Em.im, src);
  v.En.re = __shfl_sync(kFull, v.En.re, src);
  v.En.im = __shfl_sync(kFull, v.En.im, src);
  v.pre_m.re = __shfl_sync(kFull, v.pre_m.re, src);
  v.pre_m.im = __shfl_sync(kFull, v.pre_m.im, src);
  v.pre_n.re = __shfl_sync(kFull, v.pre_n.re, src);
  v.pre_n.im = __shfl_sync(kFull, v.pre_n.im, src);
#pragma unroll
  for (int j = 0; j < 3; ++j)
    v.pos[j] = __shfl_sync(kFull, v.pos[j], src);
  v.wgt = __shfl_sync(kFull, v.wgt, src);
  v.ids = __shfl_sync(kFull, v.ids, src);
  if (timed) {
    v.opath = __shfl_sync(kFull, v.opath, src);
    v.t_launch = __shfl_sync(kFull, v.t_launch, src);
  }
}

// This lane's vertex for sensor s: false when process_estimation would return before
// the bin loop (events filter, I_norm, weight; src/detector.cpp:1356-1380).  The
// interior product folds the newest event's raw factor into the committed one from
// two events on (src/detector.cpp:1462-1469), in binary64.
template <typename T, typename R>
__device__ __forceinline__ bool est_prepare(const Scene &sc, const RunParams &rp, const Photon<R> &ph,
                                            const Side<R> &side, int med_idx, const Sensor &s, EstV<T> &v)
{
  if (s.f_events && ((int)ph.events < s.events_min || (int)ph.events > s.events_max))
    return false;
  const Medium &med = sc.media[med_idx];
  if (med.I_norm < 1e-300)
    return false;
  // the layer's aggregate albedo at the first vertex (src/detector.cpp:1378), the
  // selected species' own later (:1472); the same for a HomogeneousLayer
  const Layer &VL = sc.layers[ph.layer];
  const double w_scatter = ph.w * (ph.events == 0 ? VL.mu_s / VL.mu_t : med.mu_s / med.mu_t);
  if (w_scatter < 1e-300)
    return false;
  v.wgt = sizeof(T) == 8 ? (T)w_scatter : (T)(w_scatter / (3.141592653589793 * med.I_norm));
  const int tid = threadIdx.x;
  const double px = ph.px, py = ph.py, pz = ph.pz;
  v.pos[0] = (T)px; v.pos[1] = (T)py; v.pos[2] = (T)pz;
#pragma unroll
  for (int j = 0; j < 9; ++j)
    v.P[j] = (T)ph.P[j];
  v.Em = {(T)ph.Em.re, (T)ph.Em.im};
  v.En = {(T)ph.En.re, (T)ph.En.im};
  v.opath = ph.opath;
  const bool multi = ph.events >= 1;
  v.ids = med_idx | (side.first_med[tid] << 8) | (ph.layer << 16) | ((multi ? 1 : 0) << 24);
  v.pre_m = {T(0), T(0)};
  v.pre_n = {T(0), T(0)};
  if (multi) {
    const Cx<double> T0 = {side.T[0][tid], side.T[1][tid]}, T1 = {side.T[2][tid], side.T[3][tid]};
    const Cx<double> T2 = {side.T[4][tid], side.T[5][tid]}, T3 = {side.T[6][tid], side.T[7][tid]};
    Cx<double> Td[4] = {T0, T1, T2, T3};
    if (ph.events >= 2) {
      const Cx<double> pS2 = {side.last[0][tid], side.last[1][tid]};
      const Cx<double> pS1 = {side.last[2][tid], side.last[3][tid]};
      const double pc = side.last[4][tid], ps = side.last[5][tid];
      const Cx<double> B00 = cscale(pS2, pc), B01 = cscale(pS2, ps), B10 = cscale(pS1, -ps),
                       B11 = cscale(pS1, pc);
      Td[0] = cadd(cmul(B00, T0), cmul(B01, T2));
      Td[1] = cadd(cmul(B00, T1), cmul(B01, T3));
      Td[2] = cadd(cmul(B10, T0), cmul(B11, T2));
      Td[3] = cadd(cmul(B10, T1), cmul(B11, T3));
    }
    const Cx<T> Tt[4] = {{(T)Td[0].re, (T)Td[0].im}, {(T)Td[1].re, (T)Td[1].im},
                         {(T)Td[2].re, (T)Td[2].im}, {(T)Td[3].re, (T)Td[3].im}};
    est_prefix<T>(sc, v.P, Tt, med_idx, v.pre_m, v.pre_n);
  }
  v.t_launch = (s.dt > 0) ? emission_time<R>(sc.laser, rp, ph.index()) : 0.0;
  return true;
}

// Whether a vertex at depth z > 0 in `layer` can reach the plane z = 0 with a
// transmittance of 1e-20 or more for some bin: the path to the plane is at least z
// and crosses only the layers from 0 to `layer`, so its optical depth is at least
// z times the smallest mu_t among them; e^-47 < 1e-20 leaves a margin over the
// per-bin test's rounding.
__device__ __forceinline__ bool est_reachable(const Scene &sc, double z, int layer)
{
  double mu = sc.layers[0].mu_t;
  for (int i = 1; i <= layer && i < sc.n_layers; ++i)
    mu = fmin(mu, sc.layers[i].mu_t);
  return !(mu * z > 47.0);
}

// r_1 and the frame after the first scatter of the vertex prepared by thread st,
// from its Side column; r_n - r_1 (CBS phase) formed in binary64.
template <typename T>
__device__ __forceinline__ void est_first(const Side<T> &side, int st, const T *pos, T *P1, T *dr)
{
#pragma unroll
  for (int j = 0; j < 9; ++j)
    P1[j] = side.first[3 + j][st];
#pragma unroll
  for (int j = 0; j < 3; ++j)
    dr[j] = (T)((double)pos[j] - (double)side.first[j][st]);
}

// One bin of one vertex, binary64 (FarFieldCBSSensor::process_estimation,
// src/detector.cpp:1384-1560, per bin); src_t: the thread that prepared the vertex.
__device__ __forceinline__ void est_bin(const Scene &sc, const Sensor &s, const EstV<double> &v, int b,
                                        const Side<double> &side, int src_t, const EstTarget &tg)
{
  const Laser &L = sc.laser;
  const Medium &med = sc.media[v.med()];
  const double4 bin = s.est_bins[b];
  const V3<double> s_out = v3<double>(bin.x, bin.y, bin.z);
  const double denom = s_out.z;                            // plane z = 0, normal +z
  if (fabs(denom) < 1e-14)
    return;
  const double Lp = (-v.pos[2]) / denom;
  if (Lp <= 0.0)
    return;
  const double Tr = exp(-est_optical_depth(sc, v.pos, s_out, Lp));
  if (Tr < 1e-20)
    return;
  const V3<double> m_cur = drow(v.P, 0), n_cur = drow(v.P, 1), s_cur = drow(v.P, 2);
  const V3<double> pv = vcross_unit(s_cur, s_out);
  const double pn = sqrt(vdot(pv, pv));
  if (pn < 1e-12)
    return;
  const V3<double> p_hat = vscale(pv, 1.0 / pn);
  const double sin_phi = -vdot(m_cur, p_hat);
  const double cos_phi = vdot(n_cur, p_hat);
  double cdot = vdot(s_cur, s_out);
  cdot = cdot > 1.0 ? 1.0 : (cdot < -1.0 ? -1.0 : cdot);
  const double th_scat = acos(cdot);
  Cx<double> S2, S1;
  amplitudes<double>(med, th_scat, S2, S1);
  const double s22 = cnorm(S2), s11 = cnorm(S1);
  const double Emm = cnorm(v.Em), Enn = cnorm(v.En);
  const double c2 = cos_phi * cos_phi, sn2 = sin_phi * sin_phi;
  const double e12 = v.Em.re * v.En.re + v.Em.im * v.En.im;
  const double F = Emm * (s22 * c2 + s11 * sn2) + Enn * (s22 * sn2 + s11 * c2) +
                   2.0 * e12 * (s22 - s11) * sin_phi * cos_phi;
  if (F < 1e-300)
    return;
  const double prob_bin = (F / (3.141592653589793 * med.I_norm)) * bin.w;
  const double w_bin = v.wgt * Tr * prob_bin;
  if (w_bin < 1e-300)
    return;
  const int t_idx = time_bin(s, v.t_launch + (v.opath + Lp));
  if (t_idx < 0)
    return;
  // amp = sqrt(w_bin) exp(i k L) in the reference (src/detector.cpp:1425, :1533); the
  // phase multiplies the forward and the reverse field alike and cancels in every
  // Stokes value, so only the modulus is formed
  const Cx<double> amp = {sqrt(w_bin), 0.0};
  // exit frame A(theta, phi) P (src/detector.cpp:1027-1045)
  double st, ct;
  sincos(th_scat, &st, &ct);
  double Pe[9];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const double mj = v.P[j], nj = v.P[3 + j], sj = v.P[6 + j];
    Pe[j] = ct * cos_phi * mj + ct * sin_phi * nj + (-st) * sj;
    Pe[3 + j] = -sin_phi * mj + cos_phi * nj + 0.0 * sj;
    Pe[6 + j] = st * cos_phi * mj + st * sin_phi * nj + ct * sj;
  }
  // forward field (S R(phi)) E / sqrt(F) (src/detector.cpp:121-160)
  const double inv = 1.0 / sqrt(F);
  const Cx<double> T00 = cscale(S2, cos_phi), T01 = cscale(S2, sin_phi);
  const Cx<double> T10 = cscale(S1, -sin_phi), T11 = cscale(S1, cos_phi);
  const Cx<double> Efm = cmul(cscale(cadd(cmul(T00, v.Em), cmul(T01, v.En)), inv), amp);
  const Cx<double> Efn = cmul(cscale(cadd(cmul(T10, v.Em), cmul(T11, v.En)), inv), amp);
  const Cx<double> Efx = cadd(cscale(Efm, Pe[0]), cscale(Efn, Pe[3]));
  const Cx<double> Efy = cadd(cscale(Efm, Pe[1]), cscale(Efn, Pe[4]));
  Cx<double> Erx = {0.0, 0.0}, Ery = {0.0, 0.0};
  if (v.multi()) {
    const V3<double> s_in = v3<double>(L.dir[0], L.dir[1], L.dir[2]);
    Cx<double> Rm, Rn;
    double P1[9], dr[3];
    est_first(side, src_t, v.pos, P1, dr);
    est_suffix(sc, P1, Pe, v.first_med(), v.pre_m, v.pre_n, Rm, Rn);
    const double qx = (s_out.x + s_in.x) * L.k, qy = (s_out.y + s_in.y) * L.k,
                 qz = (s_out.z + s_in.z) * L.k;
    const double arg = qx * dr[0] + qy * dr[1] + qz * dr[2];
    double sp_, cp_;
    sincos(arg, &sp_, &cp_);
    const Cx<double> pp = {cp_, sp_};
    const Cx<double> Rm2 = cmul(cmul(Rm, amp), pp), Rn2 = cmul(cmul(Rn, amp), pp);
    Erx = cadd(cscale(Rm2, Pe[0]), cscale(Rn2, Pe[3]));
    Ery = cadd(cscale(Rm2, Pe[1]), cscale(Rn2, Pe[4]));
  }
  // accumulate_stokes (src/detector.cpp:1194-1226)
  const Cx<double> Ex = cadd(Efx, Erx), Ey = cadd(Efy, Ery);
  const Cx<double> c_xy = cmul(Ex, Cx<double>{Ey.re, -Ey.im});
  const Cx<double> f_xy = cmul(Efx, Cx<double>{Efy.re, -Efy.im});
  const Cx<double> r_xy = cmul(Erx, Cx<double>{Ery.re, -Ery.im});
  const double c0 = cnorm(Ex) + cnorm(Ey), c1 = cnorm(Ex) - cnorm(Ey);
  const double c2s = 2.0 * c_xy.re, c3 = 2.0 * c_xy.im;
  const double i0 = cnorm(Efx) + cnorm(Efy) + cnorm(Erx) + cnorm(Ery);
  const double i1 = cnorm(Efx) - cnorm(Efy) + cnorm(Erx) - cnorm(Ery);
  const double i2 = 2.0 * (f_xy.re + r_xy.re), i3 = 2.0 * (f_xy.im + r_xy.im);
  const unsigned long long P = s.plane_stride;
  const unsigned long long tstride = (unsigned long long)s.N_theta * s.N_phi;
  const unsigned long long cell = (unsigned long long)b;   // bins enumerate (theta, phi) row-major
  if (!in_bounds(kBoundEst, (unsigned long long)(t_idx > 0 ? t_idx : 0) * tstride + cell < P))
    return;
  tg.add4(P, cell, c0, c1, c2s, c3);
  tg.add4(P, 4 * P + cell, i0, i1, i2, i3);
  if (t_idx >= 1) {
    tg.add4(P, t_idx * tstride + cell, c0, c1, c2s, c3);
    tg.add4(P, 4 * P + t_idx * tstride + cell, i0, i1, i2, i3);
  }
}

// The same bin in binary32 for binary32 transport (the CBS phase excepted): bin
// directions from the binary32 copy of the bin table, the scattering angle as
// atan2(|s_cur x s_out|, s_cur . s_out), binary32 amplitudes, transmittance, fields
// and Stokes values, accumulated in binary64.  The CBS phase q . (r_n - r_1) uses the
// table's q = k (s_out + s_in), formed in binary64, and r_n - r_1 formed in binary64.
__device__ __forceinline__ void est_bin_f32(const Scene &sc, const Sensor &s, const EstV<float> &v, int b,
                                            const Side<float> &side, int src_t, const EstTarget &tg)
{
  const Medium &med = sc.media[v.med()];
  const float4 *bf = reinterpret_cast<const float4 *>(s.est_bins + s.est_n);
  const float4 bin = bf[2 * b];
  const V3<float> s_out = v3<float>(bin.x, bin.y, bin.z);
  const float denom = s_out.z;                             // plane z = 0, normal +z
  if (fabsf(denom) < 1e-14f)
    return;
  const float pz = v.pos[2];
  const float Lp = -pz / denom;
  if (!(Lp > 0.f))
    return;
  const double posd[3] = {(double)v.pos[0], (double)v.pos[1], (double)v.pos[2]};
  const float tau = sc.n_layers == 1
      ? sc.layers[v.layer()].mu_t_f * Lp
      : (float)est_optical_depth(sc, posd, v3<double>(bin.x, bin.y, bin.z), (double)Lp);
  const float Tr = expf(-tau);
  if (Tr < 1e-20f)
    return;
  const V3<float> m_cur = trow<float>(v.P, 0), n_cur = trow<float>(v.P, 1), s_cur = trow<float>(v.P, 2);
  // |s_cur x s_out| = sin(theta_scat) of the two unit vectors; its direction is the
  // scattering plane's normal p_hat (vcross_unit, src/vec.cpp:14-26)
  const V3<float> pv = {s_cur.y * s_out.z - s_cur.z * s_out.y, s_cur.z * s_out.x - s_cur.x * s_out.z,
                        s_cur.x * s_out.y - s_cur.y * s_out.x};
  const float pn = sqrtf(vdot(pv, pv));
  if (!(pn > 0.f))
    return;
  const V3<float> p_hat = vscale(pv, 1.f / pn);
  const float sin_phi = -vdot(m_cur, p_hat);
  const float cos_phi = vdot(n_cur, p_hat);
  const float cdot = vdot(s_cur, s_out);
  const float th_scat = atan2f(pn, cdot);
  Cx<float> S2, S1;
  amplitudes<float>(med, th_scat, S2, S1);
  const float s22 = cnorm(S2), s11 = cnorm(S1);
  const float Emm = cnorm(v.Em), Enn = cnorm(v.En);
  const float e12 = v.Em.re * v.En.re + v.Em.im * v.En.im;
  const float c2 = cos_phi * cos_phi, sn2 = sin_phi * sin_phi;
  const float F = Emm * (s22 * c2 + s11 * sn2) + Enn * (s22 * sn2 + s11 * c2) +
                  2.f * e12 * (s22 - s11) * sin_phi * cos_phi;
  if (!(F > 0.f))
    return;
  // p(Omega) dOmega = F / (pi I_norm) x dOmega dphi; w mu_s / mu_t / (pi I_norm) in wgt
  const float w_bin = v.wgt * Tr * F * bin.w;
  if (!(w_bin > 0.f))
    return;
  const int t_idx = time_bin(s, v.t_launch + (v.opath + (double)Lp));
  if (t_idx < 0)
    return;
  const float amp = sqrtf(w_bin);
  // exit frame A(theta, phi) P (src/detector.cpp:1027-1045): cos, sin of th_scat
  const float ih = rsqrtf(cdot * cdot + pn * pn);
  const float ct = cdot * ih, st = pn * ih;
  float Pe[9];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const float mj = v.P[j], nj = v.P[3 + j], sj = v.P[6 + j];
    Pe[j] = ct * cos_phi * mj + ct * sin_phi * nj - st * sj;
    Pe[3 + j] = -sin_phi * mj + cos_phi * nj;
    Pe[6 + j] = st * cos_phi * mj + st * sin_phi * nj + ct * sj;
  }
  // forward field (S R(phi)) E / sqrt(F) (src/detector.cpp:121-160)
  const float inv = amp * rsqrtf(F);
  const Cx<float> T00 = cscale(S2, cos_phi), T01 = cscale(S2, sin_phi);
  const Cx<float> T10 = cscale(S1, -sin_phi), T11 = cscale(S1, cos_phi);
  const Cx<float> Efm = cscale(cadd(cmul(T00, v.Em), cmul(T01, v.En)), inv);
  const Cx<float> Efn = cscale(cadd(cmul(T10, v.Em), cmul(T11, v.En)), inv);
  const Cx<float> Efx = cadd(cscale(Efm, Pe[0]), cscale(Efn, Pe[3]));
  const Cx<float> Efy = cadd(cscale(Efm, Pe[1]), cscale(Efn, Pe[4]));
  Cx<float> Erx = {0.f, 0.f}, Ery = {0.f, 0.f};
  if (v.multi()) {
    Cx<float> Rm, Rn;
    float P1[9], dr[3];
    est_first(side, src_t, v.pos, P1, dr);
    est_suffix<float>(sc, P1, Pe, v.first_med(), v.pre_m, v.pre_n, Rm, Rn);
    const float4 q = bf[2 * b + 1];
    const float arg = q.x * dr[0] + q.y * dr[1] + q.z * dr[2];
    float sp_, cp_;
    sincosf(arg, &sp_, &cp_);
    const Cx<float> pp = {cp_ * amp, sp_ * amp};
    const Cx<float> Rm2 = cmul(Rm, pp), Rn2 = cmul(Rn, pp);
    Erx = cadd(cscale(Rm2, Pe[0]), cscale(Rn2, Pe[3]));
    Ery = cadd(cscale(Rm2, Pe[1]), cscale(Rn2, Pe[4]));
  }
  // accumulate_stokes (src/detector.cpp:1194-1226)
  const Cx<float> Ex = cadd(Efx, Erx), Ey = cadd(Efy, Ery);
  const Cx<float> c_xy = cmul(Ex, Cx<float>{Ey.re, -Ey.im});
  const Cx<float> f_xy = cmul(Efx, Cx<float>{Efy.re, -Efy.im});
  const Cx<float> r_xy = cmul(Erx, Cx<float>{Ery.re, -Ery.im});
  const double c0 = cnorm(Ex) + cnorm(Ey), c1 = cnorm(Ex) - cnorm(Ey);
  const double c2s = 2.0 * c_xy.re, c3 = 2.0 * c_xy.im;
  const double i0 = cnorm(Efx) + cnorm(Efy) + cnorm(Erx) + cnorm(Ery);
  const double i1 = cnorm(Efx) - cnorm(Efy) + cnorm(Erx) - cnorm(Ery);
  const double i2 = 2.0 * ((double)f_xy.re + r_xy.re), i3 = 2.0 * ((double)f_xy.im + r_xy.im);
  const unsigned long long PS = s.plane_stride;
  const unsigned long long tstride = (unsigned long long)s.N_theta * s.N_phi;
  const unsigned long long cell = (unsigned long long)b;
  if (!in_bounds(kBoundEst, (unsigned long long)(t_idx > 0 ? t_idx : 0) * tstride + cell < PS))
    return;
  tg.add4(PS, cell, c0, c1, c2s, c3);
  tg.add4(PS, 4 * PS + cell, i0, i1, i2, i3);
  if (t_idx >= 1) {
    tg.add4(PS, t_idx * tstride + cell, c0, c1, c2s, c3);
    tg.add4(PS, 4 * PS + t_idx * tstride + cell, i0, i1, i2, i3);
  }
}

// The lane of the (k+1)-th set bit of mask (k < popc(mask)): the smallest b with
// popc(mask & bits 0..b) > k, by binary search on b.
__device__ __forceinline__ int nth_set_lane(unsigned mask, int k)
{
  int lo = 0, hi = 31;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const unsigned upto = (mid == 31) ? 0xffffffffu : ((2u << mid) - 1u);
    if (__popc(mask & upto) > k)
      hi = mid;
    else
      lo = mid + 1;
  }
  return lo;
}

// run_estimators (src/detector.cpp:274-281, called at src/simulation.cpp:419-426) for
// the whole warp: `at` marks the lanes whose photon is at a vertex in medium med_idx.
// Every lane of the warp calls it (converged).  Vertices are estimated in binary64 by
// binary64 transport and in binary32 (CBS phase and tallies binary64) by binary32
// transport, with two ways of dealing the (vertex, bin) pairs out to the lanes:
//  * binary32: the warp's vertices are broadcast one at a time and lane j takes bins
//    j, j + 32, ... of each (the vertex stays in registers over its bins);
//  * binary64: the pairs of all the warp's vertices are numbered vertex-major and lane
//    j takes pairs j, j + 32, ...: in each step a lane fetches the vertex of its own
//    pair from the lane that prepared it (a shuffle whose source differs from lane to
//    lane), which leaves no lane idle at the end of a vertex's bins.
// Each measured faster for its precision (mie_cbs_small, 100 bins: binary32 1.22 M
// against 1.16 M photons/s, binary64 0.45 M against 0.41 M).  Within a step the lanes'
// bins are distinct when the grid has 32 bins or more, so a warp's private grid copy
// takes plain adds; a smaller grid adds atomically under the flattened numbering.
template <typename R>
__device__ __noinline__ void estimate_warp(const Scene &sc, const RunParams &rp, const Photon<R> &ph,
                                           const Side<R> &side, int med_idx, bool at,
                                           unsigned long long *s_hits, double *s_est)
{
  using T = R;
  const unsigned lane = threadIdx.x & 31u;
  const int warp0 = (int)(threadIdx.x & ~31u);
  for (int si = 0; si < sc.n_sensors; ++si) {
    const Sensor &s = sc.sensors[si];
    if (s.kind != LMC_SENSOR_FARFIELD_CBS || !s.estimator)
      continue;
    EstV<T> v;
    const bool want = at && est_prepare<T, R>(sc, rp, ph, side, med_idx, s, v);
    const unsigned counted = __ballot_sync(kFull, want);
    if (lane == 0 && counted)
      atomicAdd(s_hits + si, (unsigned long long)__popc(counted));
    const bool reach = want && est_reachable(sc, (double)v.pos[2], v.layer());
    const unsigned verts = __ballot_sync(kFull, reach);
    if (!verts)
      continue;
    EstTarget tg = est_target(rp, s, si, s_est);
    const int nb = s.est_n;
    const bool timed = s.dt > 0;
    __syncwarp();                        // the lanes' Side columns, read across the warp
    if constexpr (sizeof(T) == 4) {
      for (unsigned pend = verts; pend; pend &= pend - 1u) {
        const int src = __ffs(pend) - 1;
        EstV<T> w = v;
        est_fetch(w, src, timed);
        for (int b = (int)lane; b < nb; b += 32)
          est_bin_f32(sc, s, w, b, side, warp0 + src, tg);
      }
    } else {
      if (nb < 32)
        tg.atomic = true;                // two pairs of a step may share a bin
      const int pairs = __popc(verts) * nb;
      for (int p0 = 0; p0 < pairs; p0 += 32) {
        const int p = p0 + (int)lane;
        const int k = p < pairs ? p / nb : 0;             // the vertex of this lane's pair
        const int src = nth_set_lane(verts, k);           // its preparing lane
        EstV<T> w = v;
        est_fetch(w, src, timed);
        if (p < pairs)
          est_bin(sc, s, w, p - k * nb, side, warp0 + src, tg);
      }
    }
  }
}

// Sensor::check_conditions (src/detector.cpp:374-417)
template <typename R>
__device__ __forceinline__ bool check_conditions(const Sensor &s, double hx, double hy, const Photon<R> &ph,
                                                 int crossing)
{
  if (s.f_dir && s.direction != 2 && s.direction != crossing)
    return false;
  if (s.f_events && ((int)ph.events < s.events_min || (int)ph.events > s.events_max))
    return false;
  if (s.f_theta) {
    double d[3];
    exit_dir(ph.P[6], ph.P[7], ph.P[8], d);
    const double ct = -1.0 * d[2];
    if (ct < s.cos_min || ct > s.cos_max)
      return false;
  }
  if (s.f_phi) {
    double phi = atan2((double)ph.P[7], (double)ph.P[6]);
    if (phi < 0)
      phi += 2.0 * 3.141592653589793;
    if (phi < s.phi_min || phi > s.phi_max)
      return false;
  }
  if (s.f_pos) {
    if (hx < s.x_min || hx > s.x_max || hy < s.y_min || hy > s.y_max)
      return false;
  }
  return true;
}

// The frame before the newest scatter, P_{n-1} = A(theta_n, phi_n)^T P_n (A is a
// rotation), from the newest scatter's angles; the launch frame before any scatter.
template <typename R>
__device__ __forceinline__ void prev_frame(const Photon<R> &ph, const Side<R> &side, R *out)
{
  const int tid = threadIdx.x;
  if (ph.events == 0) {
#pragma unroll
    for (int j = 0; j < 9; ++j)
      out[j] = ph.P[j];
    return;
  }
  const R ct = side.ang[0][tid], st = side.ang[1][tid];
  const R cp = side.ang[2][tid], sp = side.ang[3][tid];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const R m = ph.P[j], n = ph.P[3 + j], s = ph.P[6 + j];
    out[j] = ct * cp * m - sp * n + st * cp * s;
    out[3 + j] = ct * sp * m + cp * n + st * sp * s;
    out[6 + j] = -st * m + ct * s;
  }
}

template <typename R>
__device__ __forceinline__ void fill_hit(const Photon<R> &ph, const Side<R> &side, R hx, R hy, R hz,
                                         double opath, HitData<R> &h)
{
  const int tid = threadIdx.x;
  h.p_lo = ph.rng.p_lo;
  h.p_hi = ph.rng.p_hi;
  h.events = ph.events;
  h.first_med = side.first_med[tid];
  h.last_med = ph.last_med;
  h.w = ph.w;
  h.opath = opath;
  h.pen = (double)ph.pen;
  h.hx = hx; h.hy = hy; h.hz = hz;
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    h.P[j] = ph.P[j];
    h.P1[j] = side.first[3 + j][tid];
  }
  prev_frame<R>(ph, side, h.Pn1);
  h.Em = ph.Em;
  h.En = ph.En;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    h.r1[j] = side.first[j][tid];
    h.rn[j] = side.rn[j][tid];
  }
#pragma unroll
  for (int q = 0; q < 4; ++q)
    h.T[q] = {side.T[2 * q][tid], side.T[2 * q + 1][tid]};
}

// Whether a hit's FarFieldCBS sensors will read its reverse-path fields: from the
// second scattering event on (src/detector.cpp:1290) and when the exit direction falls
// in one of their grids (the binning of hit_farfield, src/detector.cpp:1271-1281),
// widened by a bin on every side so that no hit a grid bins is missed.
template <typename R>
__device__ __forceinline__ bool needs_reverse(const Scene &sc, unsigned mask, const Photon<R> &ph)
{
  const unsigned m = mask & sc.cbs_mask;
  if (!m || ph.events < 2)
    return false;
  const R theta = exit_theta(ph.P[6], ph.P[7], ph.P[8]);
  R phi = m_atan2(ph.P[7], ph.P[6]);
  if (phi < R(0))
    phi += R(6.283185307179586);
  for (int si = 0; si < sc.n_sensors; ++si) {
    if (!(m & (1u << si)))
      continue;
    const Sensor &s = sc.sensors[si];
    const int it = (int)(theta / R(s.dtheta)), jp = (int)(phi / R(s.dphi));
    if (it >= -1 && it <= s.N_theta && jp >= -1 && jp <= s.N_phi)
      return true;
  }
  return false;
}

// Append a hit to the queue (warp-aggregated slot).  Only the fields the
// sensors in `mask` read are written.
template <typename R, bool kAdj>
__device__ __forceinline__ void enqueue_hit(const Scene &sc, const RunParams &rp, const Photon<R> &ph,
                                            const Side<R> &side, const Flight<R> &fl, R t,
                                            R hx, R hy, R hz, double opath, unsigned mask)
{
  const unsigned active = __activemask();
  const unsigned lane = threadIdx.x & 31u;
  const int leader = __ffs(active) - 1;
  unsigned long long base = 0;
  if ((int)lane == leader)
    base = atomicAdd(&rp.scratch->queue_count, (unsigned long long)__popc(active));
  base = __shfl_sync(active, base, leader);
  const unsigned long long slot = base + __popc(active & ((1u << lane) - 1u));
  const Queue &q = rp.queue;
  if (slot >= q.cap) {
    atomicOr(&rp.scratch->error_flags, (unsigned)kErrQueueOverflow);
    return;
  }
  const int tid = threadIdx.x;
  const unsigned long long C = q.cap;
  q.u32[kQPhotonLo * C + slot] = ph.rng.p_lo;
  q.u32[kQPhotonHi * C + slot] = ph.rng.p_hi;
  q.u32[kQEvents * C + slot] = ph.events;
  q.u32[kQMask * C + slot] = mask;
  q.u32[kQMedia * C + slot] = (uint32_t)side.first_med[tid] | ((uint32_t)ph.last_med << 16);
  q.u32[kQScene * C + slot] = (uint32_t)ph.scene;
  q.f64[kQWeight * C + slot] = ph.w;
  q.f64[kQOpath * C + slot] = opath;
  if (mask & sc.stat_mask)
    q.f64[kQPen * C + slot] = (double)ph.pen;
  R *r = static_cast<R *>(q.r);
  r[(kQHit + 0) * C + slot] = hx;
  r[(kQHit + 1) * C + slot] = hy;
  r[(kQHit + 2) * C + slot] = hz;
#pragma unroll
  for (int j = 0; j < 9; ++j)
    r[(kQP + j) * C + slot] = ph.P[j];
  r[(kQE + 0) * C + slot] = ph.Em.re;
  r[(kQE + 1) * C + slot] = ph.Em.im;
  r[(kQE + 2) * C + slot] = ph.En.re;
  r[(kQE + 3) * C + slot] = ph.En.im;
  if ((mask & sc.cbs_mask) && rp.cbs_replay) {
    // no history kept: the replay kernel rebuilds it for the hits a grid will read
    if (needs_reverse<R>(sc, mask, ph)) {
      const unsigned long long k = atomicAdd(&rp.scratch->replay_count, 1ull);
      if (k < C)
        rp.replay_list[k] = (uint32_t)slot;
    }
  } else if (mask & sc.cbs_mask) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      r[(kQR1 + j) * C + slot] = side.first[j][tid];
      r[(kQRn + j) * C + slot] = side.rn[j][tid];
    }
    R pn1[9];
    prev_frame<R>(ph, side, pn1);
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      r[(kQP1 + j) * C + slot] = side.first[3 + j][tid];
      r[(kQPn1 + j) * C + slot] = pn1[j];
    }
#pragma unroll
    for (int qd = 0; qd < 4; ++qd) {
      r[(kQT + 2 * qd) * C + slot] = side.T[2 * qd][tid];
      r[(kQT + 2 * qd + 1) * C + slot] = side.T[2 * qd + 1][tid];
    }
  }
  if (kAdj)
    for (int k = 0; k < rp.adj_K; ++k)
      r[(kQScore + k) * C + slot] = flight_hit_score<R>(sc, fl, t, k);
}

// SensorsGroup::record_hit (src/detector.cpp:178-270) for the step (x0,y0,z0) -> pos.
// kQueue: hits are appended to the queue for the tally kernel; otherwise they are
// processed here.  Returns whether an absorbing sensor took the photon.
template <typename R, bool kQueue, bool kAdj>
__device__ __forceinline__ bool record_hit(const Scene &sc, const RunParams &rp, Photon<R> &ph,
                                           const Side<R> &side, const Flight<R> &fl, R x0, R y0, R z0,
                                           unsigned long long *s_hits)
{
  const R z1 = z0, z2 = ph.pz;
  const int crossing = (z2 > z1) ? 0 : 1;
  const R zmin = z1 < z2 ? z1 : z2, zmax = z1 < z2 ? z2 : z1;
  bool killed = false;
  for (int g = 0; g < sc.n_planes; ++g) {
    const R zp = sc_plane<R>(sc, g);
    if (!(zp >= zmin && zp <= zmax))
      continue;
    const R dx = ph.px - x0, dy = ph.py - y0, dz = z2 - z1;
    const R t = (zp - z1) / dz;
    const R hx = x0 + dx * t, hy = y0 + dy * t, hz = z1 + dz * t;
    const R ex = hx - ph.px, ey = hy - ph.py, ez = hz - ph.pz;
    const R corr = m_sqrt(ex * ex + ey * ey + ez * ez);
    const double opath = ph.opath - (corr > R(0) ? (double)corr : 0.0);
    unsigned mask = 0;
    for (int si = 0; si < sc.n_sensors; ++si) {
      const Sensor &s = sc.sensors[si];
      if (s.plane != g || s.estimator)
        continue;
      if (!check_conditions<R>(s, (double)hx, (double)hy, ph, crossing))
        continue;
      mask |= 1u << si;
      if (s.absorb)
        killed = true;
    }
    if (mask) {
      if (kQueue) {
        enqueue_hit<R, kAdj>(sc, rp, ph, side, fl, t, hx, hy, hz, opath, mask);
      } else {
        HitData<R> h;
        fill_hit<R>(ph, side, hx, hy, hz, opath, h);
        process_hits<R, false>(sc, rp, h, mask, s_hits, nullptr, nullptr, nullptr);
      }
    }
  }
  return killed;
}

template <typename R>
__device__ void init_photon(const Scene &sc, const RunParams &rp, Photon<R> &ph, Side<R> &side,
                            unsigned long long index)
{
  const Laser &L = sc.laser;
  rng_reset(ph.rng, index);
  double x, y, t;
  source_sample<R>(L, ph.rng, rp, x, y, t);
  ph.px = R(x);
  ph.py = R(y);
  ph.pz = R(L.pos[2]);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    ph.P[j] = R(L.m[j]);
    ph.P[3 + j] = R(L.n[j]);
    ph.P[6 + j] = R(L.dir[j]);
  }
  ph.Em = {R(L.E[0]), R(L.E[1])};
  ph.En = {R(L.E[2]), R(L.E[3])};
  ph.w = 1.0;
  ph.pen = R(0);
  ph.opath = 0.0;
  ph.events = 0;
  ph.scene = 0;
  ph.layer = layer_index_at<R>(sc, ph.pz);
  ph.last_med = 0;
  const int tid = threadIdx.x;
  side.first_med[tid] = 0;
  if (!rp.track_reverse)                                    // no history in this launch
    return;
  side.rn[0][tid] = ph.px; side.rn[1][tid] = ph.py; side.rn[2][tid] = ph.pz;   // r_1 = r_n = launch
#pragma unroll
  for (int q = 0; q < 8; ++q)
    side.T[q][tid] = R(q == 0 || q == 6 ? 1 : 0);
  side.first[0][tid] = ph.px; side.first[1][tid] = ph.py; side.first[2][tid] = ph.pz;
#pragma unroll
  for (int j = 0; j < 9; ++j)
    side.first[3 + j][tid] = ph.P[j];                       // P1 = P0
}

enum Fate { kAlive = 0, kDetected = 1, kEscaped = 2, kStack = 3, kRoulette = 4, kCap = 5, kError = 6 };

// Upper bound on azimuth rejection trials per event.  The acceptance rate is
// >= 1/2 for any finite (S, E) (F(phi) averages (a+b)/2 >= Fmax/2), so this is
// only reached when the state is not finite; the photon is then dropped and
// the run reports kErrAborted instead of spinning.
constexpr int kMaxRejectionTrials = 1 << 16;

// Absorption::record_absorption (src/absortion.cpp:54-91): an event's deposit at the
// photon's position (x, y, z), into slice 0 and, time-resolved, into the slice of its
// arrival time t.  Out of line and with scalar arguments, so that the photon state
// stays in registers: only scenes with an Absorption recorder reach it.
__device__ __noinline__ void record_absorption(const AbsorbGrid &g, double *tallies, double x, double y,
                                               double z, double t, double d_weight)
{
  const double r = sqrt(x * x + y * y);
  if (!(r <= g.radius) || !(z >= 0.0) || !(z <= g.depth))
    return;
  const double fr = floor(r / g.d_r), fz = floor(z / g.d_z);
  if (!(fr < (double)g.n_r) || !(fz < (double)g.n_z))
    return;
  const unsigned long long cell = (unsigned long long)fr * (unsigned long long)g.n_z +
                                  (unsigned long long)fz;
  double *grid = tallies + g.off;
  if (!in_bounds(kBoundAbsorb, cell < (unsigned long long)g.n_r * (unsigned long long)g.n_z))
    return;
  atomicAdd(grid + cell, d_weight);
  if (g.d_t > 0.0) {
    const double fk = floor(t / g.d_t) + 1.0;
    if (fk >= 1.0 && fk < (double)g.n_t)
      atomicAdd(grid + (unsigned long long)fk * (unsigned long long)g.n_r * (unsigned long long)g.n_z + cell,
                d_weight);
  }
}

// The same deposit for the binary32 transport: the cell from the binary32 position by
// reciprocal multiplies instead of binary64 divisions.  The position itself carries
// binary32 rounding (~1e-7 relative), so the bin edges are no blurrier than the position.
// Short enough to inline into the binary32 transport.
__device__ __forceinline__ void record_absorption_f32(const AbsorbGrid &g, double *tallies, float x,
                                                   float y, float z, double t, double d_weight)
{
  const float r = sqrtf(x * x + y * y);
  if (!(r <= g.radius_f) || !(z >= 0.0f) || !(z <= g.depth_f))
    return;
  const float fr = floorf(r * g.inv_dr_f), fz = floorf(z * g.inv_dz_f);
  if (!(fr < (float)g.n_r) || !(fz < (float)g.n_z))
    return;
  const unsigned long long cell = (unsigned long long)fr * (unsigned long long)g.n_z +
                                  (unsigned long long)fz;
  double *grid = tallies + g.off;
  if (!in_bounds(kBoundAbsorb, cell < (unsigned long long)g.n_r * (unsigned long long)g.n_z))
    return;
  atomicAdd(grid + cell, d_weight);
  if (g.d_t > 0.0) {
    const double fk = floor(t / g.d_t) + 1.0;
    if (fk >= 1.0 && fk < (double)g.n_t)
      atomicAdd(grid + (unsigned long long)fk * (unsigned long long)g.n_r * (unsigned long long)g.n_z + cell,
                d_weight);
  }
}

// First half of one loop iteration of run_photon (src/simulation.cpp:297-426): the
// free flight with its interface crossings and sensor planes, the inside test and the
// scattering species.  Returns the photon's fate; kAlive leaves the photon at its next
// scattering vertex, in medium med_out.
// kExtras: the MixtureLayer species draw and the Absorption recorder are compiled in
// (scenes without either run the variant without their code).  kHits = false (the CBS
// replay) leaves the sensor planes out: a replayed event never reaches one, because
// crossing a plane at z <= 0 ends a photon.
template <typename R, bool kQueue, bool kAdj, bool kExtras = false, bool kHits = true>
__device__ __forceinline__ int event_move(const Scene &sc, const RunParams &rp, Photon<R> &ph,
                                          Side<R> &side, Flight<R> &fl, Counters &cnt,
                                          unsigned long long *s_hits, int &med_out)
{
  rng_prefetch<R>(ph.rng, rp);
  {
    // free path with the layer's mean free path (src/medium.cpp:123-126,
    // src/sample.cpp:90-94)
    R step = -lay_mfp<R>(sc.layers[ph.layer]) * m_log(uniform<R>(ph.rng, rp));
    cnt.steps++;
    if (kAdj)
      flight_start<R>(sc, fl, sc.layers[ph.layer].medium);
    const R dx = ph.P[6], dy = ph.P[7], dz = ph.P[8];
    // Move to the next interface (src/simulation.cpp:318-382) or by the whole
    // step (:389-400), testing the sensor planes after each move (:355, :403).
    for (int crossing = 0;; ++crossing) {
      bool at_iface = false;
      R zi = R(0), s_move = step;
      if (sc.n_interfaces > 0 && find_next_interface<R>(sc, ph.pz, ph.pz + dz * step, zi)) {
        const R dz_total = dz * step;
        if (fabs(dz_total) >= R(1e-15)) {
          const R t = (zi - ph.pz) / dz_total;
          if (t >= R(0) && t <= R(1)) {
            at_iface = true;
            s_move = step * t;
          }
        }
      }
      if (at_iface && crossing >= sc.n_interfaces)   // each crossing passes a distinct interface
        return kError;
      const R rem = at_iface ? (step - s_move) * lay_mut<R>(sc.layers[ph.layer]) : R(0);
      ph.opath += (double)s_move;
      const R x0 = ph.px, y0 = ph.py, z0 = ph.pz;
      ph.px += dx * s_move;
      ph.py += dy * s_move;
      if (at_iface) {
        ph.pz = m_nudge(zi + ((dz > R(0)) ? R(1e-12) : R(-1e-12)), zi, dz > R(0));
      } else {
        ph.pz += dz * s_move;
        if (ph.pz > ph.pen)
          ph.pen = ph.pz;
      }
      if (kAdj) {
        fl.seg_med = sc.layers[ph.layer].medium;
        fl.seg_len = s_move;
      }
      if (kHits && sc.n_planes > 0 && fabs(ph.pz - z0) >= R(1e-12)) {
        const R zlo = z0 < ph.pz ? z0 : ph.pz, zhi = z0 < ph.pz ? ph.pz : z0;
        if (sc_plane<R>(sc, 0) <= zhi && sc_plane<R>(sc, sc.n_planes - 1) >= zlo &&
            record_hit<R, kQueue, kAdj>(sc, rp, ph, side, fl, x0, y0, z0, s_hits))
          return kDetected;
      }
      if (!at_iface)
        break;
      if (kAdj)
        flight_segment_done<R>(sc, fl, fl.seg_med, s_move);
      const int nl = layer_index_at<R>(sc, ph.pz);
      if (nl >= sc.n_layers)
        return kStack;
      ph.layer = nl;
      const R nmt = lay_mut<R>(sc.layers[nl]);
      step = (nmt > R(0)) ? rem / nmt : rem;
    }
    // Sample::is_inside (src/sample.cpp:268-288)
    if (!(isfinite(ph.px) && isfinite(ph.py) && isfinite(ph.pz)) || ph.pz < R(0) ||
        (!sc.top_is_inf && ph.pz >= sc_top<R>(sc)))
      return kEscaped;
  }
  ph.layer = layer_index_at<R>(sc, ph.pz);
  // Layer::select_scatter_medium (src/simulation.cpp:419-425): a HomogeneousLayer's
  // medium without a draw, or a MixtureLayer species by one uniform and lower_bound
  // on its selection CDF (src/sample.cpp:96-104), compared in binary64
  const Layer &SL = sc.layers[ph.layer];
  const int lflags = SL.flags;
  int med_idx = SL.medium;
  if (kExtras && (lflags & kLayerMixture)) {
    const double u = (double)uniform<R>(ph.rng, rp);
    int i = 0;
    while (i < SL.n_species - 1 && sc.mix_cdf[SL.mix_begin + i] < u)
      ++i;
    med_idx = sc.mix_species[SL.mix_begin + i];
  }
  if (kAdj)
    flight_scatter<R>(sc, fl, fl.seg_med, fl.seg_len);
  med_out = med_idx;
  return kAlive;
}

// Second half (src/simulation.cpp:429-613): the scatter at the vertex in medium med_idx
// (theta, S(theta), the conditional azimuth, frame, Jones vector, CBS bookkeeping), the
// absorption weight, roulette and the event cap.  kDeposit = false (the CBS replay)
// leaves the Absorption recorder out: the transport recorded those deposits already.
template <typename R, bool kAdj, bool kExtras = false, bool kDeposit = true>
__device__ __forceinline__ int event_scatter(const Scene &sc, const RunParams &rp, Photon<R> &ph,
                                             Side<R> &side, Flight<R> &fl, Counters &cnt, int med_idx)
{
  const Layer &SL = sc.layers[ph.layer];
  const int lflags = SL.flags;
  const Medium &m = sc.media[med_idx];
  const R theta = sample_theta<R>(m, uniform<R>(ph.rng, rp));  // :429
  Cx<R> S2, S1;
  amplitudes<R>(m, theta, S2, S1);                            // :430
  // sample_phi_conditional (src/phase.cpp:27-49)
  const R s2sq = cnorm(S2), s1sq = cnorm(S1);
  const R e1sq = cnorm(ph.Em), e2sq = cnorm(ph.En);
  const R e12 = ph.Em.re * ph.En.re + ph.Em.im * ph.En.im;
  const R a = s2sq * e1sq + s1sq * e2sq;
  const R b = s1sq * e1sq + s2sq * e2sq;
  const R c = R(2) * (s2sq - s1sq) * e12;
  const R diff = a - b;
  const R Fmax = R(0.5) * (a + b) + R(0.5) * m_sqrt(diff * diff + c * c);
  // The first kSpecTrials trials are evaluated together, from numbers the ring
  // already holds, and the first accepted one is taken with only the draws up to it
  // consumed: the same phi and the same stream position as trial-by-trial
  // rejection, without a loop whose trip count differs from lane to lane.  Lanes
  // that reject them all (or whose ring is short, at a photon's first event)
  // continue one trial at a time.
  R cp = R(1), sp = R(0);
  R Facc = R(1);                 // F(phi) of the accepted trial (> 0: u > 0 accepted it)
  int trial = 0;
  {
    constexpr int kSpec = sizeof(R) == 4 ? 3 : 2;
    const uint32_t wpd = words_per_draw<R>(rp);
    if (ph.rng.filled >= (ph.rng.draw + 2u * kSpec) * wpd) {
      bool acc = false;
      uint32_t take = 2u * kSpec;
#pragma unroll 1                  // rolled: a smaller event loop for the instruction cache
      for (int t = 0; t < kSpec; ++t) {
        const R u1 = peek_uniform<R>(ph.rng, rp, 2u * t);
        const R u2 = peek_uniform<R>(ph.rng, rp, 2u * t + 1u);
        R st_, ct_;
        m_sincos_turn(u1, &st_, &ct_);
        const R F = a * ct_ * ct_ + b * st_ * st_ + c * ct_ * st_;
        const R Fc = F > R(0) ? F : R(0);
        if (!acc && u2 * Fmax <= Fc) {
          cp = ct_;
          sp = st_;
          Facc = F;
          take = 2u * t + 2u;
          acc = true;
        }
      }
      ph.rng.draw += take;
      trial = acc ? -1 : kSpec;
    }
  }
  if (trial >= 0) {
    for (;; ++trial) {
      if (trial == kMaxRejectionTrials)
        return kError;
      const R u1 = uniform<R>(ph.rng, rp);
      m_sincos_turn(u1, &sp, &cp);
      const R F = a * cp * cp + b * sp * sp + c * cp * sp;
      const R Fc = F > R(0) ? F : R(0);
      Facc = F;
      if (uniform<R>(ph.rng, rp) * Fmax <= Fc)
        break;
    }
  }
  R st, ct;
  m_sincos(theta, &st, &ct);
  if (kAdj)
    flight_event<R>(sc, fl, med_idx, ct);
  // frame update P <- A(theta, phi) P (src/simulation.cpp:438-453); P_{n-1} <- old P
  if (rp.track_reverse) {              // the newest scatter's angles (P_{n-1} = A^T P_n)
    const int tid = threadIdx.x;
    side.ang[0][tid] = ct;
    side.ang[1][tid] = st;
    side.ang[2][tid] = cp;
    side.ang[3][tid] = sp;
  }
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const R mj = ph.P[j], nj = ph.P[3 + j], sj = ph.P[6 + j];
    ph.P[j] = ct * cp * mj + ct * sp * nj - st * sj;
    ph.P[3 + j] = -sp * mj + cp * nj;
    ph.P[6 + j] = st * cp * mj + st * sp * nj + ct * sj;
  }
  // Jones update E <- (S R(phi)) E / sqrt(F) (src/simulation.cpp:456-492); F(phi)
  // is the density the rejection step just evaluated (the same quadratic form)
  {
    const Cx<R> Em = ph.Em, En = ph.En;
    const R inv = R(1) / m_sqrt(Facc);
    const Cx<R> T00 = cscale(S2, cp * inv), T01 = cscale(S2, sp * inv);
    const Cx<R> T10 = cscale(S1, -sp * inv), T11 = cscale(S1, cp * inv);
    ph.Em = cadd(cmul(T00, Em), cmul(T01, En));
    ph.En = cadd(cmul(T10, Em), cmul(T11, En));
  }
  if (rp.track_reverse) {                                     // :495-568
    const int tid = threadIdx.x;
    const uint32_t evt = ph.events + 1;
    if (evt == 1) {
      side.first[0][tid] = ph.px; side.first[1][tid] = ph.py; side.first[2][tid] = ph.pz;
#pragma unroll
      for (int j = 0; j < 9; ++j)
        side.first[3 + j][tid] = ph.P[j];
      side.first_med[tid] = med_idx;
    }
    side.rn[0][tid] = ph.px; side.rn[1][tid] = ph.py; side.rn[2][tid] = ph.pz;
    ph.last_med = med_idx;
    if (evt >= 3) {
      // T <- J_{n-1} T, J_{n-1} = diag(S2, S1) R(phi) of the previous event: the real
      // rotation first, then the rows scaled by S2 and S1.  The reference renormalises
      // T (Frobenius) at every event only to stay in range; every use of T ends in a
      // normalised field, so its scale is free, and every fourth event suffices for
      // binary32's range (|S| products over three events stay far inside it).
      const Cx<R> pS2 = {side.last[0][tid], side.last[1][tid]};
      const Cx<R> pS1 = {side.last[2][tid], side.last[3][tid]};
      const R pc = side.last[4][tid], ps = side.last[5][tid];
      const Cx<R> T0 = {side.T[0][tid], side.T[1][tid]}, T1 = {side.T[2][tid], side.T[3][tid]};
      const Cx<R> T2 = {side.T[4][tid], side.T[5][tid]}, T3 = {side.T[6][tid], side.T[7][tid]};
      const Cx<R> u0 = cadd(cscale(T0, pc), cscale(T2, ps)), u1 = cadd(cscale(T1, pc), cscale(T3, ps));
      const Cx<R> u2 = cadd(cscale(T2, pc), cscale(T0, -ps)), u3 = cadd(cscale(T3, pc), cscale(T1, -ps));
      Cx<R> t0 = cmul(pS2, u0), t1 = cmul(pS2, u1), t2 = cmul(pS1, u2), t3 = cmul(pS1, u3);
      if ((evt & 3u) == 0u) {
        const R frob = m_sqrt(cnorm(t0) + cnorm(t1) + cnorm(t2) + cnorm(t3));
        if (frob > tiny<R>()) {
          const R inv = R(1) / frob;
          t0 = cscale(t0, inv); t1 = cscale(t1, inv); t2 = cscale(t2, inv); t3 = cscale(t3, inv);
        }
      }
      side.T[0][tid] = t0.re; side.T[1][tid] = t0.im; side.T[2][tid] = t1.re; side.T[3][tid] = t1.im;
      side.T[4][tid] = t2.re; side.T[5][tid] = t2.im; side.T[6][tid] = t3.re; side.T[7][tid] = t3.im;
    }
    if (evt >= 2) {
      side.last[0][tid] = S2.re; side.last[1][tid] = S2.im;
      side.last[2][tid] = S1.re; side.last[3][tid] = S1.im;
      side.last[4][tid] = cp; side.last[5][tid] = sp;
    }
  }
  ph.events++;                                                // :578-587
  cnt.events++;
  if (kExtras && kDeposit && (lflags & kLayerAbsorb)) {       // :589-592
    const double t = sc.absorb.d_t > 0.0 ? launch_time<R>(sc, rp, ph) + ph.opath : 0.0;  // velocity 1
    const double dw = SL.mu_t > 0 ? ph.w * SL.absorb_prob : 1.0;
    if constexpr (std::is_same<R, float>::value)
      record_absorption_f32(sc.absorb, rp.tallies, ph.px, ph.py, ph.pz, t, dw);
    else
      record_absorption(sc.absorb, rp.tallies, (double)ph.px, (double)ph.py, (double)ph.pz, t, dw);
  }
  ph.w *= SL.albedo;                                          // the layer's aggregate albedo
  if (ph.w < 1e-4) {                                          // :596-607
    if (uniform<R>(ph.rng, rp) < R(0.1))
      ph.w /= 0.1;
    else
      return kRoulette;
  }
  if ((int)ph.events > rp.max_events)                         // :609-613
    return kCap;
  return kAlive;
}

// One loop iteration of run_photon (src/simulation.cpp:297-614).  Returns the photon's
// fate (kAlive if it continues).
template <typename R, bool kQueue, bool kAdj, bool kExtras = false>
__device__ __forceinline__ int event_step(const Scene &sc, const RunParams &rp, Photon<R> &ph,
                                          Side<R> &side, Flight<R> &fl, Counters &cnt,
                                          unsigned long long *s_hits)
{
  int med_idx = 0;
  const int fate = event_move<R, kQueue, kAdj, kExtras>(sc, rp, ph, side, fl, cnt, s_hits, med_idx);
  if (fate != kAlive)
    return fate;
  return event_scatter<R, kAdj, kExtras>(sc, rp, ph, side, fl, cnt, med_idx);
}

template <typename R>
__device__ void write_record(const Scene &sc, const RunParams &rp, const Photon<R> &ph,
                             const Side<R> &side, int fate)
{
  const int tid = threadIdx.x;
  lmc_record &r = rp.records[ph.index() - rp.photon_begin];
  r.photon = ph.index();
  r.events = ph.events;
  r.draws = ph.rng.draw;
  r.fate = fate;
  r.layer = ph.layer;
  r.weight = ph.w;
  r.opticalpath = ph.opath;
  r.penetration_depth = ph.pen;
  r.launch_time = launch_time<R>(sc, rp, ph);
  r.pos[0] = ph.px; r.pos[1] = ph.py; r.pos[2] = ph.pz;
  for (int j = 0; j < 3; ++j) {
    r.m[j] = ph.P[j];
    r.n[j] = ph.P[3 + j];
    r.dir[j] = ph.P[6 + j];
    r.r1[j] = side.first[j][tid];
    r.rn[j] = side.rn[j][tid];
  }
  r.E[0] = ph.Em.re; r.E[1] = ph.Em.im; r.E[2] = ph.En.re; r.E[3] = ph.En.im;
}

// Copy the scene into shared memory (every thread reads it every event).
__device__ __forceinline__ void load_scene(unsigned char *s_raw, const Scene *g_scene)
{
  const int4 *src = reinterpret_cast<const int4 *>(g_scene);
  int4 *dst = reinterpret_cast<int4 *>(s_raw);
  for (int i = threadIdx.x; i < (int)(sizeof(Scene) / 16); i += blockDim.x)
    dst[i] = src[i];
}

// Amplitude tables into shared memory (1-D bulk copies by the tensor memory accelerator,
// completion counted on an mbarrier; the source is this GPU's own table arena).  Thread
// 0 issues one cp.async.bulk per medium -- sizes and both addresses are multiples of 16
// bytes, which the arena's 256-byte alignment and 16-byte table entries guarantee --
// and waits with a bounded number of tries; the block's scene copy then points each
// medium at its staged table.  A copy that does not complete in time raises kErrStaging
// and leaves the scene on the global tables.
__device__ __forceinline__ void stage_amplitudes(Scene &sc, const RunParams &rp, unsigned char *s_dyn,
                                                 unsigned long long *mbar)
{
  if (threadIdx.x == 0) {
    const unsigned bar = (unsigned)__cvta_generic_to_shared(mbar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(rp.stage_bytes)
                 : "memory");
    unsigned off = rp.stage_off;
    for (int m = 0; m < sc.n_media; ++m) {
      const unsigned bytes = (unsigned)sc.media[m].amp_n * 16u;
      const unsigned dst = (unsigned)__cvta_generic_to_shared(s_dyn + off);
      asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                   ::"r"(dst), "l"(sc.media[m].amp_f), "r"(bytes), "r"(bar) : "memory");
      off += bytes;
    }
    bool done = false;
    for (int tries = 0; tries < (1 << 22) && !done; ++tries) {
      unsigned ok;
      asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
                   " selp.u32 %0, 1, 0, p;\n}" : "=r"(ok) : "r"(bar) : "memory");
      done = ok != 0;
    }
    if (done) {
      off = rp.stage_off;
      for (int m = 0; m < sc.n_media; ++m) {
        sc.media[m].amp_stage = reinterpret_cast<const float4 *>(s_dyn + off);
        off += (unsigned)sc.media[m].amp_n * 16u;
      }
    } else {
      atomicOr(&rp.scratch->error_flags, (unsigned)kErrStaging);
    }
  }
}

// kMinBlocks > 1 asks the compiler to fit that many 256-thread blocks per SM
// (register cap 65536 / (256 kMinBlocks)); lmc_run picks the variant.

// Scene of global photon g in a sweep: the s with prefix[s] <= g < prefix[s + 1].
__device__ __forceinline__ int sweep_scene(const RunParams &rp, unsigned long long g)
{
  int lo = 0, hi = rp.n_scenes - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (rp.sweep_prefix[mid] <= g)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// kEst: the scene has an estimator-mode FarFieldCBS sensor (estimate_warp at every
// vertex).  kAdj: likelihood-ratio run (queued mode only).  kSweep: g_scene is an array of
// rp.n_scenes scenes read from global memory (L1-cached), photon g belongs to scene
// sweep_scene(g), and each lane follows its own photon's scene.
template <typename R, bool kQueue, int kMinBlocks, bool kAdj = false, bool kSweep = false, bool kEst = false,
          bool kExtras = false>
__global__ void __launch_bounds__(kBlock, kMinBlocks) transport_kernel(const Scene *__restrict__ g_scene, RunParams rp)
{
  __shared__ __align__(16) unsigned char s_raw[kSweep ? 16 : sizeof(Scene)];
  __shared__ unsigned long long s_hits[LMC_MAX_SENSORS];
  __shared__ unsigned long long s_fate[7];
  extern __shared__ __align__(16) unsigned char s_dyn[];
  Side<R> &side = *reinterpret_cast<Side<R> *>(s_dyn);
  Flight<R> fl;
  fl.score = reinterpret_cast<R *>(s_dyn + rp.side_off) + threadIdx.x;
  if (!kSweep)
    load_scene(s_raw, g_scene);
  if (threadIdx.x < LMC_MAX_SENSORS)
    s_hits[threadIdx.x] = 0;
  if (threadIdx.x < 7)
    s_fate[threadIdx.x] = 0;
  double *s_est = reinterpret_cast<double *>(s_dyn + rp.side_off);
  if (kEst)
    for (int j = threadIdx.x; j < rp.est_smem_doubles; j += blockDim.x)
      s_est[j] = 0.0;
  __syncthreads();
  if (!kSweep && sizeof(R) == 4 && rp.stage_bytes) {
    __shared__ __align__(8) unsigned long long s_mbar;
    stage_amplitudes(*reinterpret_cast<Scene *>(s_raw), rp, s_dyn, &s_mbar);
    __syncthreads();
  }
  const Scene *scp = kSweep ? g_scene : reinterpret_cast<const Scene *>(s_raw);
  const unsigned lane = threadIdx.x & 31u;
  Counters cnt = {0, 0, 0};
  Photon<R> ph;
  ph.rng.ring = &side.ring[0][threadIdx.x];
  bool alive = false, done = false;
  for (;;) {
    const unsigned need = __ballot_sync(kFull, !alive && !done);
    if (need) {
      const int leader = __ffs(need) - 1;
      unsigned long long base = 0;
      if ((int)lane == leader)
        base = atomicAdd(&rp.scratch->next_photon, (unsigned long long)__popc(need));
      base = __shfl_sync(kFull, base, leader);
      if (!alive && !done) {
        const unsigned long long idx = base + __popc(need & ((1u << lane) - 1u));
        if (idx < rp.n_photons) {
          int si = 0;
          if (kSweep) {
            si = sweep_scene(rp, rp.photon_begin + idx);
            scp = g_scene + si;
          }
          init_photon<R>(*scp, rp, ph, side, rp.photon_begin + idx);
          ph.scene = si;
          if (kAdj)
            for (int k = 0; k < rp.adj_K; ++k)
              fl[k] = R(0);
          alive = true;
        } else {
          done = true;
        }
      }
    }
    if (__all_sync(kFull, done))
      break;
    int fate = kAlive;
    if constexpr (kEst) {
      // the move, then the warp's estimate at the vertices reached (all lanes, converged),
      // then the scatter
      int med_idx = 0;
      if (alive)
        fate = event_move<R, kQueue, kAdj, kExtras>(*scp, rp, ph, side, fl, cnt, s_hits, med_idx);
      estimate_warp<R>(*scp, rp, ph, side, med_idx, alive && fate == kAlive, s_hits, s_est);
      if (alive && fate == kAlive)
        fate = event_scatter<R, kAdj, kExtras>(*scp, rp, ph, side, fl, cnt, med_idx);
    } else if (alive) {
      fate = event_step<R, kQueue, kAdj, kExtras>(*scp, rp, ph, side, fl, cnt, s_hits);
    }
    if (alive) {
      if (fate != kAlive) {
        alive = false;
        cnt.draws += ph.rng.draw;
        atomicAdd(&s_fate[fate], 1ull);
        if (rp.records)
          write_record<R>(*scp, rp, ph, side, fate);
        if (fate == kError)
          atomicOr(&rp.scratch->error_flags, (unsigned)kErrAborted);
        if (!isfinite(ph.w))
          atomicOr(&rp.scratch->error_flags, (unsigned)kErrNonFiniteWeight);
      }
    }
  }
  // warp-reduce the per-thread counters, then one atomic per warp
  unsigned long long ev = cnt.events, st = cnt.steps, dr = cnt.draws;
  for (int o = 16; o > 0; o >>= 1) {
    ev += __shfl_down_sync(kFull, ev, o);
    st += __shfl_down_sync(kFull, st, o);
    dr += __shfl_down_sync(kFull, dr, o);
  }
  if (lane == 0) {
    atomicAdd(&rp.scratch->events, ev);
    atomicAdd(&rp.scratch->steps, st);
    atomicAdd(&rp.scratch->draws, dr);
  }
  __syncthreads();
  if (threadIdx.x < LMC_MAX_SENSORS && s_hits[threadIdx.x])
    atomicAdd(&rp.scratch->hits[threadIdx.x], s_hits[threadIdx.x]);
  if (threadIdx.x == kError && s_fate[kError])
    atomicAdd(&rp.scratch->photons, s_fate[kError]);
  if (threadIdx.x >= 1 && threadIdx.x < 6 && s_fate[threadIdx.x]) {
    unsigned long long *dst = threadIdx.x == kDetected ? &rp.scratch->detected
                              : threadIdx.x == kEscaped ? &rp.scratch->escaped
                              : threadIdx.x == kStack   ? &rp.scratch->stack
                              : threadIdx.x == kRoulette ? &rp.scratch->roulette
                                                         : &rp.scratch->cap;
    atomicAdd(dst, s_fate[threadIdx.x]);
    atomicAdd(&rp.scratch->photons, s_fate[threadIdx.x]);
  }
  if (kEst && rp.est_smem_doubles > 0) {      // the block's estimated grids into the tallies
    const Scene &sc = *scp;
    const int copies = rp.est_per_warp ? (int)(blockDim.x >> 5) : 1;
    for (int si = 0; si < sc.n_sensors; ++si) {
      const int o = rp.est_smem[si];
      if (o < 0)
        continue;
      const Sensor &s = sc.sensors[si];
      const int n = (int)(8 * s.plane_stride);
      for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double v = 0.0;
        for (int w = 0; w < copies; ++w)
          v += s_est[w * rp.est_warp_doubles + o + j];
        if (v != 0.0)
          atomicAdd(rp.tallies + s.tally_off + j, v);
      }
    }
  }
}

// CBS replay kernel: for every hit on the replay list, re-run the photon from its
// launch -- the same stream (seed, photon index), the same transport code -- through its
// recorded number of scattering events with the reverse-path bookkeeping on, and write
// the CBS fields (r_1, r_n, P_1, P_{n-1}, the interior product T, the first and last
// species) into its queue entry, where the tally kernel reads them.  The replay must
// reach the recorded hit state: the frame and Jones vector after the last event are
// compared with the entry's, and a replay that does not match, or whose photon ends
// early, raises kErrReplay.  Persistent like the transport: each loop iteration advances
// every busy lane by one event, and a lane whose replay is finished takes the next list
// entry from a shared counter (warp-aggregated), so a warp never waits for the longest
// of 32 replays that were handed out together.
template <typename R, bool kSweep = false, bool kExtras = false>
__global__ void __launch_bounds__(kBlock, sizeof(R) == 4 ? 3 : 2)
    cbs_replay_kernel(const Scene *__restrict__ g_scene, RunParams rp)
{
  __shared__ __align__(16) unsigned char s_raw[kSweep ? 16 : sizeof(Scene)];
  extern __shared__ __align__(16) unsigned char s_dyn[];
  Side<R> &side = *reinterpret_cast<Side<R> *>(s_dyn);
  if (!kSweep)
    load_scene(s_raw, g_scene);
  __syncthreads();
  const Queue &q = rp.queue;
  const unsigned long long C = q.cap;
  const unsigned long long listed = *(volatile unsigned long long *)&rp.scratch->replay_count;
  const unsigned long long n = listed < C ? listed : C;
  if (blockIdx.x == 0 && threadIdx.x == 0)
    atomicAdd(&rp.scratch->replayed, n);
  rp.track_reverse = 1;
  const unsigned lane = threadIdx.x & 31u;
  const int tid = threadIdx.x;
  Photon<R> ph;
  ph.rng.ring = &side.ring[0][threadIdx.x];
  Flight<R> fl;
  fl.score = nullptr;
  Counters cnt = {0, 0, 0};
  R *r = static_cast<R *>(q.r);
  const Scene *scp = kSweep ? g_scene : reinterpret_cast<const Scene *>(s_raw);
  unsigned long long slot = 0;
  uint32_t target = 0;
  bool busy = false, done = false;
  for (;;) {
    const unsigned need = __ballot_sync(kFull, !busy && !done);
    if (need) {
      const int leader = __ffs(need) - 1;
      unsigned long long base = 0;
      if ((int)lane == leader)
        base = atomicAdd(&rp.scratch->replay_next, (unsigned long long)__popc(need));
      base = __shfl_sync(kFull, base, leader);
      if (!busy && !done) {
        const unsigned long long i = base + __popc(need & ((1u << lane) - 1u));
        if (i < n) {
          slot = rp.replay_list[i];
          if (kSweep)
            scp = g_scene + q.u32[kQScene * C + slot];
          const unsigned long long index =
              ((unsigned long long)q.u32[kQPhotonHi * C + slot] << 32) | q.u32[kQPhotonLo * C + slot];
          target = q.u32[kQEvents * C + slot];
          init_photon<R>(*scp, rp, ph, side, index);
          busy = true;
        } else {
          done = true;
        }
      }
    }
    if (__all_sync(kFull, done))
      break;
    if (!busy)
      continue;
    if (ph.events < target) {                    // one more event of this replay
      int med = 0;
      int fate = event_move<R, true, false, kExtras, false>(*scp, rp, ph, side, fl, cnt, nullptr, med);
      if (fate == kAlive)
        fate = event_scatter<R, false, kExtras, false>(*scp, rp, ph, side, fl, cnt, med);
      if (fate != kAlive) {                      // ended before its recorded hit
        atomicOr(&rp.scratch->error_flags, (unsigned)kErrReplay);
        busy = false;
      }
      continue;
    }
    busy = false;
    // the frame and Jones vector of the hit are those after the last scatter
    R dev = R(0);
#pragma unroll
    for (int j = 0; j < 9; ++j)
      dev = fmax(dev, fabs(ph.P[j] - r[(kQP + j) * C + slot]));
    dev = fmax(dev, fabs(ph.Em.re - r[(kQE + 0) * C + slot]));
    dev = fmax(dev, fabs(ph.Em.im - r[(kQE + 1) * C + slot]));
    dev = fmax(dev, fabs(ph.En.re - r[(kQE + 2) * C + slot]));
    dev = fmax(dev, fabs(ph.En.im - r[(kQE + 3) * C + slot]));
    if (ph.events != target || !(dev <= R(1e-3))) {
      atomicOr(&rp.scratch->error_flags, (unsigned)kErrReplay);
      continue;
    }
    q.u32[kQMedia * C + slot] = (uint32_t)side.first_med[tid] | ((uint32_t)ph.last_med << 16);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      r[(kQR1 + j) * C + slot] = side.first[j][tid];
      r[(kQRn + j) * C + slot] = side.rn[j][tid];
    }
    R pn1[9];
    prev_frame<R>(ph, side, pn1);
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      r[(kQP1 + j) * C + slot] = side.first[3 + j][tid];
      r[(kQPn1 + j) * C + slot] = pn1[j];
    }
#pragma unroll
    for (int qd = 0; qd < 8; ++qd)
      r[(kQT + qd) * C + slot] = side.T[qd][tid];
  }
}

// Tally kernel: one thread per queued hit runs the sensors' process_hit.
// kAdj: also the likelihood-ratio outputs; the radial ones are summed per block in
// (1 + adj_K) * (adj_radial_bins + 1) doubles of dynamic shared memory.
// kSweep: each entry carries its scene (an index into the g_scene array) and hit
// counts go to rp.sweep_hits.
// kT (lmc_tally_mode less one): kTallyWarp combines the adds of a warp's lanes into
// one cell; kTallyShared (one scene) gives the block private copies of the grids
// rp.tally_smem names, after the radial outputs in dynamic shared memory: zeroed
// here, added to with shared atomics, and added into the tallies when the block ends.
// Binary32 kernels (but a sweep's with likelihood-ratio scores) are held to 128
// registers, so that two blocks (16 warps) fit per SM: the kernel is latency-bound
// (shared-memory, SFU and queue-read waits), and 154 registers left 8 warps per SM.
template <typename R, bool kAdj = false, bool kSweep = false, int kT = kTallyGlobal>
__global__ void __launch_bounds__(kBlock, (sizeof(R) == 4 && !(kAdj && kSweep)) ? 2 : 1)
    tally_kernel(const Scene *__restrict__ g_scene, RunParams rp)
{
  static_assert(!(kSweep && kT == kTallyShared), "private grids hold one scene");
  __shared__ __align__(16) unsigned char s_raw[kSweep ? 16 : sizeof(Scene)];
  __shared__ unsigned long long s_hits[LMC_MAX_SENSORS];
  extern __shared__ __align__(16) unsigned char s_dyn[];
  double *s_rad = reinterpret_cast<double *>(s_dyn);
  // radial outputs in shared memory (one scene per launch); a sweep adds them globally
  const int rad_n = (kAdj && !kSweep && rp.adj_radial_sensor >= 0)
                        ? (1 + rp.adj_K) * (rp.adj_radial_bins + 1) : 0;
  if (!kSweep)
    load_scene(s_raw, g_scene);
  if (threadIdx.x < LMC_MAX_SENSORS)
    s_hits[threadIdx.x] = 0;
  for (int j = threadIdx.x; j < rad_n; j += blockDim.x)
    s_rad[j] = 0.0;
  double *const priv = (kT == kTallyShared) ? s_rad + rad_n : nullptr;
  if (kT == kTallyShared)
    for (int j = threadIdx.x; j < rp.tally_smem_doubles; j += blockDim.x)
      priv[j] = 0.0;
  __syncthreads();
  const Scene &sc0 = *reinterpret_cast<const Scene *>(s_raw);
  const Queue &q = rp.queue;
  const unsigned long long C = q.cap;
  const unsigned long long count = *(volatile unsigned long long *)&rp.scratch->queue_count;
  const unsigned long long n = count < C ? count : C;
  const R *r = static_cast<const R *>(q.r);
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned scene = kSweep ? q.u32[kQScene * C + i] : 0u;
    const Scene &sc = kSweep ? g_scene[scene] : sc0;
    HitData<R> h;
    h.p_lo = q.u32[kQPhotonLo * C + i];
    h.p_hi = q.u32[kQPhotonHi * C + i];
    h.events = q.u32[kQEvents * C + i];
    const unsigned mask = q.u32[kQMask * C + i];
    const uint32_t media = q.u32[kQMedia * C + i];
    h.first_med = media & 0xffffu;
    h.last_med = media >> 16;
    h.w = q.f64[kQWeight * C + i];
    h.opath = q.f64[kQOpath * C + i];
    h.pen = (mask & sc.stat_mask) ? q.f64[kQPen * C + i] : 0.0;
    h.hx = r[(kQHit + 0) * C + i];
    h.hy = r[(kQHit + 1) * C + i];
    h.hz = r[(kQHit + 2) * C + i];
#pragma unroll
    for (int j = 0; j < 9; ++j)
      h.P[j] = r[(kQP + j) * C + i];
    h.Em = {r[(kQE + 0) * C + i], r[(kQE + 1) * C + i]};
    h.En = {r[(kQE + 2) * C + i], r[(kQE + 3) * C + i]};
    if (mask & sc.cbs_mask) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        h.r1[j] = r[(kQR1 + j) * C + i];
        h.rn[j] = r[(kQRn + j) * C + i];
      }
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        h.P1[j] = r[(kQP1 + j) * C + i];
        h.Pn1[j] = r[(kQPn1 + j) * C + i];
      }
#pragma unroll
      for (int qd = 0; qd < 4; ++qd)
        h.T[qd] = {r[(kQT + 2 * qd) * C + i], r[(kQT + 2 * qd + 1) * C + i]};
    }
    R hs[kAdj ? kAdjMaxK : 1];
    AdjView A;
    if (kAdj) {
      A = adj_view<kSweep>(rp, scene);
      for (int k = 0; k < A.K; ++k)
        hs[k] = r[(kQScore + k) * C + i];
    }
    process_hits<R, kAdj, kT>(sc, rp, h, mask,
                              kSweep ? rp.sweep_hits + (unsigned long long)scene * LMC_MAX_SENSORS : s_hits,
                              hs, rad_n ? s_rad : nullptr, kAdj ? &A : nullptr, priv);
  }
  __syncthreads();
  if (kT == kTallyShared) {              // the block's private grids into the tallies
    for (int si = 0; si < sc0.n_sensors; ++si) {
      const int o = rp.tally_smem[si];
      if (o < 0)
        continue;
      double *dst = rp.tallies + sc0.sensors[si].tally_off;
      for (int j = threadIdx.x; j < rp.tally_smem_n[si]; j += blockDim.x) {
        const double v = priv[o + j];
        if (v != 0.0)
          atomicAdd(dst + j, v);
      }
    }
  }
  if (threadIdx.x < LMC_MAX_SENSORS && s_hits[threadIdx.x])
    atomicAdd(&rp.scratch->hits[threadIdx.x], s_hits[threadIdx.x]);
  if (kAdj && rad_n) {                   // radial outputs sit at offset 0 of every row
    const int row = rp.adj_radial_bins + 1;
    for (int j = threadIdx.x; j < rad_n; j += blockDim.x)
      if (s_rad[j] != 0.0)
        atomicAdd(rp.adj_out + (unsigned long long)(j / row) * rp.adj_n_out + (j % row), s_rad[j]);
  }
}

// Backward contraction of the likelihood-ratio outputs: grad[k] = sum_j
// J[(1 + k) n_out + j] g[j].  One block per parameter, fixed-order tree reduction,
// so the result does not depend on scheduling.
__global__ void __launch_bounds__(kBlock) adjoint_contract_kernel(const double *__restrict__ J,
                                                                  const double *__restrict__ g,
                                                                  unsigned long long n_out,
                                                                  double *__restrict__ grad)
{
  __shared__ double s[kBlock];
  const double *row = J + (unsigned long long)(1 + blockIdx.x) * n_out;
  double acc = 0.0;
  for (unsigned long long j = threadIdx.x; j < n_out; j += blockDim.x)
    acc = fma(row[j], g[j], acc);
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    grad[blockIdx.x] = s[0];
}

}  // namespace dev
}  // namespace lmc
