// oracle/replay_rng.cpp -- TEST INFRASTRUCTURE (the oracle's replay seam).
//
// Drop-in replacement for the reference's src/rng.cpp (src/rng.cpp:5-27),
// linked with the reference's other, unmodified sources by oracle/Makefile
// (target `replay`).  The reference re-seeds its generator once per photon
// index, `rng.seed_state(mix_seed(config.seed, i))` (src/simulation.cpp:197),
// and `mix_seed`, `Rng::uniform` and `Rng::normal` are defined out of line
// (include/luminis/math/rng.hpp:38,87-88).  Replacing those three definitions
// makes the unmodified transport (run_photon, sensors, laser, media) consume
// the counter-based Philox stream of oracle/philox_ref.h keyed by
// (seed, photon index, draw index) -- the stream the GPU kernel draws.
//
// mix_seed still returns the reference's SplitMix finaliser so seed_state()
// behaves as before; it additionally records (seed, photon) in thread-local
// state and rewinds the draw counter.  Thread-local state keeps the replay
// correct for any n_threads, as the reference's own per-photon seeding is.
#include <luminis/math/rng.hpp>

#include <cmath>
#include <cstdint>

#include "philox_ref.h"

namespace {
thread_local std::uint64_t tl_seed = 0;
thread_local std::uint64_t tl_photon = 0;
thread_local std::uint64_t tl_draw = 0;
int g_format = LMC_STREAM_U53;
}  // namespace

extern "C" __attribute__((visibility("default"))) void lmc_replay_set_format(int format)
{
  g_format = format;
}

extern "C" __attribute__((visibility("default"))) int lmc_replay_get_format(void)
{
  return g_format;
}

namespace luminis::math {

std::uint64_t mix_seed(std::uint64_t base, std::uint64_t tid)
{
  tl_seed = base;
  tl_photon = tid;
  tl_draw = 0;
  std::uint64_t z = base + 0x9E3779B97F4A7C15ULL * (tid + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

double Rng::uniform()
{
  return lmc_ref_stream_uniform(tl_seed, tl_photon, tl_draw++, g_format);
}

// Same Box-Muller form as src/rng.cpp:18-27, drawing from the replay stream.
double Rng::normal(const double mean, const double stddev)
{
  double u1 = uniform();
  while (u1 <= 0.0)
    u1 = uniform();
  const double u2 = uniform();
  const double z0 = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
  return z0 * stddev + mean;
}

}  // namespace luminis::math
