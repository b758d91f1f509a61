// lmc_device.cuh -- device-side data layout and math of the transport kernel.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "luminis_b200.h"

namespace lmc {
namespace dev {

constexpr int kGuideBuckets = 4096;     // inverse-CDF guide table size (power of two)

// Bounds-checked builds (LMC_BOUNDS_CHECK, libluminis_b200_checked.so from
// `build.py --bounds-check`): every table and tally index is checked before use.  A failed
// check sets its site's bit in g_bounds_failed and the access is clamped (tables) or
// skipped (tallies); the run then fails with LMC_ERR_KERNEL naming the sites.  Product
// builds compile the checks out.
enum BoundSite {
  kBoundGuide = 0,            // guide-table bucket of an inverse-CDF search
  kBoundCdf = 1,              // node index found by the search
  kBoundAmp = 2,              // amplitude-table node of S(theta)
  kBoundFarfield = 3,         // FarFieldCBS / far-field fluence cell
  kBoundFluence = 4,          // PlanarFluence cell
  kBoundField = 5,            // PlanarField cell
  kBoundAbsorb = 6,           // Absorption grid cell
  kBoundEst = 7,              // estimator-mode FarFieldCBS cell
};
#ifdef LMC_BOUNDS_CHECK
static __device__ unsigned g_bounds_failed;
__device__ __forceinline__ bool in_bounds(int site, bool ok)
{
  if (!ok)
    atomicOr(&g_bounds_failed, 1u << site);
  return ok;
}
#else
__device__ __forceinline__ bool in_bounds(int, bool) { return true; }
#endif

// One medium as the kernel sees it.  Tables live in the handle's device arena.
struct Medium {
  int theta_kind, theta_n, amp_n, pad;
  double hg_g;
  double amp_inv_dx;
  double mu_t, mfp;                     // the medium's own (species albedo, scores)
  float hg_g_f, amp_inv_dx_f, mu_t_f, mfp_f;
  const double *th_val_d, *th_cdf_d;
  const double2 *th_cs;                  // (cdf[i], slope into node i) for the fp32 path
  const int *guide_d;                    // kGuideBuckets + 1 entries
  const double4 *amp_d;                  // (s1.re, s1.im, s2.re, s2.im) per node
  const float4 *amp_f;
  double mu_s;                           // scattering coefficient (likelihood-ratio scores)
  float mu_s_f, pad_s;
  double I_norm;                         // int (|S1|^2 + |S2|^2) sin(theta), the estimator's p(Omega)
  const float4 *amp_stage;               // the block's shared-memory copy of amp_f (null: none)
};

// A layer with its transport coefficients (Layer::mu_attenuation, mu_scattering,
// sample_free_path): its medium's for a HomogeneousLayer, the MixtureLayer aggregates
// otherwise (src/sample.cpp:41-94).  A mixture's species and selection CDF are the
// entries [mix_begin, mix_begin + n_species) of Scene::mix_cdf / mix_species.
enum LayerFlag { kLayerMixture = 1, kLayerAbsorb = 2 };   // Layer::flags

struct Layer {
  double z_min, z_max;
  int medium;                            // HomogeneousLayer: its medium
  int n_species;                         // 0: HomogeneousLayer; else MixtureLayer species
  int mix_begin;
  int flags;                             // kLayerMixture; kLayerAbsorb (the scene records)
  double mu_s, mu_t, mfp, albedo;        // albedo = mu_s / mu_t (1 if mu_t == 0: no split)
  double absorb_prob;                    // mu_a / mu_t: the weight an event deposits
  float mu_t_f, mfp_f;
};

// Absorption recorder grid (src/absortion.cpp:13-32): [n_t][n_r][n_z] doubles at
// `off` in the tally buffer.
struct AbsorbGrid {
  int on, n_t, n_r, n_z;
  double radius, depth, d_r, d_z, d_t;
  unsigned long long off;
  float radius_f, depth_f, inv_dr_f, inv_dz_f;   // binary32 transport's cell lookup
};

// StatisticsSensor histograms (src/detector.cpp:1720-1888): bin parameters and the
// offsets (doubles) of the histograms present from the sensor's tally_off.
struct StatHist {
  int set, n_events, n_theta, n_phi, n_depth, n_time, n_weight, pad;
  double theta_min, theta_max, phi_min, phi_max, depth_max, weight_max;
  double dtheta, dphi, ddepth, dtime, dweight;
  unsigned long long off[6];             // events, theta, phi, depth, time, weight
};

struct Sensor {
  int kind, plane, absorb, estimator;
  int f_theta, f_phi, f_pos, f_dir, f_events, direction, events_min, events_max;
  double cos_min, cos_max, phi_min, phi_max, x_min, x_max, y_min, y_max;
  double len_x, len_y, len_t, dx, dy, dt, dtheta, dphi;
  int N_t, N_x, N_y, N_theta, N_phi;
  int est_n;                             // estimator-mode FarFieldCBS: bins estimated
  unsigned long long tally_off;          // offset in doubles into the tally buffer
  unsigned long long plane_stride;       // doubles between Stokes planes
  union {                                // device memory, by kind:
    const double4 *est_bins;             //  estimator FarFieldCBS: per bin s_out, dOmega dphi
    const StatHist *stat;                //  StatisticsSensor: its histograms
  };
};

struct Laser {
  double pos[3], dir[3], m[3], n[3];
  double E[4];
  double k;                              // 2 pi / vacuum wavelength
  double sigma;
  int source, temporal;
  double pulse_duration, repetition_rate, time_offset;
};

// Everything the kernel needs except the per-run options; copied to shared
// memory by every block at start-up.
struct __align__(16) Scene {
  int n_layers, n_interfaces, n_media, n_sensors, n_planes, top_is_inf;
  int need_phase;                        // a PlanarField sensor needs exp(i k L)
  unsigned cbs_mask;                     // sensors whose hits need the CBS fields
  double top;                            // z_max of the last layer
  double n_step;                         // 1 / light_speed = 1 / (1 / n_host)
  double interfaces[LMC_MAX_LAYERS];
  double plane_z[LMC_MAX_SENSORS];
  float interfaces_f[LMC_MAX_LAYERS];
  float plane_z_f[LMC_MAX_SENSORS];
  float top_f, pad_f;
  Layer layers[LMC_MAX_LAYERS];
  double mix_cdf[LMC_MAX_MIX_ENTRIES];   // MixtureLayer selection CDFs (last entry 1)
  int mix_species[LMC_MAX_MIX_ENTRIES];  // MixtureLayer species (media indices)
  Medium media[LMC_MAX_MEDIA];
  Sensor sensors[LMC_MAX_SENSORS];
  Laser laser;
  AbsorbGrid absorb;
  unsigned stat_mask;                    // StatisticsSensors (hits carry the penetration depth)
};

// Device scratch of one run: photon work counter, statistics, error word.
struct Scratch {
  unsigned long long next_photon;        // reset per batch
  unsigned long long queue_count;        // reset per batch
  unsigned long long replay_count;       // reset per batch: entries of RunParams::replay_list
  unsigned long long replay_next;        // reset per batch: the replay kernel's next list entry
  unsigned long long photons, events, steps, detected, escaped, stack, roulette, cap, draws;
  unsigned long long hits[LMC_MAX_SENSORS];
  unsigned long long replayed;           // CBS replays over the run's batches
  unsigned int error_flags;
  unsigned int pad;
};

// Hit queue: one entry per (photon, crossed sensor plane) whose sensors pass their
// filters, written by the transport kernel and consumed by the tally kernel.
// Struct-of-arrays, `cap` entries per field.
enum QueueU32 { kQPhotonLo = 0, kQPhotonHi, kQEvents, kQMask, kQMedia, kQScene, kQU32Fields };
enum QueueF64 { kQWeight = 0, kQOpath, kQPen, kQF64Fields };
enum QueueR {
  kQHit = 0,                  // 3: hit point
  kQP = 3,                    // 9: P_local at the crossing (rows m, n, s)
  kQE = 12,                   // 4: Jones vector (m.re, m.im, n.re, n.im)
  kQR1 = 16,                  // 3: r_1           -- CBS fields from here on
  kQRn = 19,                  // 3: r_n
  kQP1 = 22,                  // 9: frame after the first scatter
  kQPn1 = 31,                 // 9: frame before the newest scatter
  kQT = 40,                   // 8: interior Jones product (re, im) x 4
  kQRFields = 48,
  kQRBasic = 16               // fields every entry carries
};

// Likelihood-ratio ("adjoint") runs append the photon's score, one R per parameter
// (mu_a, mu_s, mean free path, HG g of each medium), after the R fields above.
constexpr int kQScore = kQRFields;
constexpr int kAdjMaxMedia = 4;
constexpr int kAdjMaxK = 4 * kAdjMaxMedia;
constexpr int kAdjMaxRadialBins = 512;

struct Queue {
  unsigned long long cap;
  uint32_t *u32;                         // [kQU32Fields][cap]
  double *f64;                           // [kQF64Fields][cap]
  void *r;                               // R[kQRFields][cap]
};

enum ErrorFlag : unsigned int {
  kErrNonFiniteWeight = 1u << 0,   // a photon ended with a NaN/inf weight
  kErrAborted = 1u << 1,           // a photon was dropped: non-finite state (see kError)
  kErrQueueOverflow = 1u << 2,     // more hits than the queue holds (tallies incomplete)
  kErrReplay = 1u << 3,            // a replayed history did not reach its recorded hit
  kErrStaging = 1u << 4,           // a table copy into shared memory did not complete in time
};

// Likelihood-ratio output layout of one scene of a sweep: its block of (1 + K) rows of
// n_out doubles starts at out_off in RunParams::adj_out.
struct AdjScene {
  unsigned long long out_off, n_out;
  int K, radial_sensor, radial_bins, pad;
  double radial_max;
  unsigned long long cbs_off[LMC_MAX_SENSORS];
};

struct RunParams {
  unsigned long long photon_begin, n_photons;
  uint32_t key0, key1;
  int max_events, track_reverse;
  double *tallies;
  lmc_record *records;                   // this launch's photons: photon_begin + i at records[i]
  Scratch *scratch;
  Queue queue;                           // used by the queued kernel pair
  unsigned int cbs_mask;                 // sensors whose hits need the CBS fields
  unsigned int pad;
  // likelihood-ratio outputs: (1 + adj_K) rows of adj_n_out doubles; row 0 the
  // outputs, row 1 + k their derivative for parameter k = 4 medium + (mu_a, mu_s, mfp, g)
  double *adj_out;
  unsigned long long adj_n_out;
  int adj_K, adj_radial_sensor, adj_radial_bins, adj_pad;
  double adj_radial_max;
  unsigned long long adj_cbs_off[LMC_MAX_SENSORS];
  int stream_u24;                        // binary64 transport drawing u24 values
  int n_scenes;                          // sweep: scenes in the launch
  // sweep: photon g belongs to scene s with sweep_prefix[s] <= g < sweep_prefix[s + 1];
  // hit counts per scene and sensor in sweep_hits[s * LMC_MAX_SENSORS + sensor]
  const unsigned long long *sweep_prefix;
  unsigned long long *sweep_hits;
  // sweep with likelihood-ratio outputs: per-scene layouts (adj_K above is the largest K)
  const AdjScene *adj_scenes;
  // estimator-mode FarFieldCBS grids accumulated per block in shared memory: sensor i's
  // copy at est_smem[i] doubles into the block's grid area (-1: global atomics)
  // est_per_warp: each warp of the block has its own copy of those grids, est_warp_doubles
  // apart (the block's est_smem_doubles = warps x est_warp_doubles)
  int est_smem[LMC_MAX_SENSORS];
  int est_smem_doubles;
  int est_per_warp, est_warp_doubles;
  // CBS replay: the transport keeps no reverse-path history (track_reverse 0 in its
  // launch); hits a FarFieldCBS grid will read append their queue slot to replay_list,
  // and the replay kernel rebuilds those photons' histories from their streams
  int cbs_replay;
  int cbs_phase_f32;                     // the CBS geometric phase in binary32 (precision study)
  uint32_t *replay_list;
  // amplitude tables staged per block: every medium's amp_f, one after another, copied
  // by cp.async.bulk into dynamic shared memory at byte stage_off (0 bytes: not staged)
  unsigned int stage_bytes, stage_off;
  // bytes of dynamic shared memory before the likelihood-ratio scores / estimated grids:
  // the whole Side, or only its ring and first species when the run replays CBS hits
  unsigned int side_off, side_pad;
  // tally kernel, LMC_TALLY_SHARED: sensor i's grid has a block-private copy at
  // tally_smem[i] doubles into the block's private area (-1: global atomics), of
  // tally_smem_n[i] doubles; the area holds tally_smem_doubles
  int tally_smem[LMC_MAX_SENSORS];
  int tally_smem_n[LMC_MAX_SENSORS];
  int tally_smem_doubles, tally_pad;
};

}  // namespace dev
}  // namespace lmc
