/*
 * luminis_b200.h -- C ABI of the B200 photon-propagation library
 * (luminis-mc_b200/luminis_mc_b200/lib/libluminis_b200.so).
 *
 * This is the drop-in boundary for luminis-mc's photon-propagation path.  It
 * replaces the work behind the reference's Python entry point
 *   luminis_mc.run_simulation_parallel(config)   (python/python_module.cpp:664-673)
 * i.e. run_simulation_parallel(const SimConfig&)  (include/luminis/core/simulation.hpp:127,
 *                                                  src/simulation.cpp:105-249)
 * with one persistent CUDA kernel on an sm_100a GPU.  All signatures use plain C
 * types, pointers and sizes; nothing here depends on PyTorch.
 *
 * Lifecycle: lmc_create (uploads the scene and its tables, allocates the
 * handle's device scratch) -> lmc_run / lmc_run_host (any number of times) ->
 * lmc_destroy.  A handle owns one CUDA stream; calls on one handle must not
 * overlap (the same rule as the reference, which is not re-entrant on one
 * SensorsGroup).  Different handles may be used from different threads.
 *
 * Errors: every call returns lmc_status; LMC_ERR_INVALID corresponds to the
 * reference's std::invalid_argument (ValueError in Python), and the message is
 * available from lmc_last_error (thread-local).
 *
 * Random stream contract (shared with the CPU replay oracle): Philox4x32-10,
 * key = (seed lo, seed hi), counter = (block, 0, photon lo, photon hi).
 * LMC_PRECISION_FP64 draws "u53" values (2 per block, u = (2*(w>>12)+1)*2^-53 for
 * the 64-bit words x1:x0 and x3:x2); LMC_PRECISION_FP32 draws "u24" values
 * (4 per block, u = (2*(x_i>>9)+1)*2^-24).  Draw j of photon i uses block j/2
 * (u53) or j/4 (u24), in the reference's draw order (src/simulation.cpp:305-598,
 * src/phase.cpp:27-49, src/laser.cpp:11-99).
 */
#ifndef LUMINIS_B200_H
#define LUMINIS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LMC_ABI_VERSION 1

#if defined(__GNUC__)
#define LMC_API __attribute__((visibility("default")))
#else
#define LMC_API
#endif
#define LMC_MAX_LAYERS 16
#define LMC_MAX_MEDIA 16
#define LMC_MAX_SENSORS 8
#define LMC_MAX_SPECIES 8         /* co-located species of one MixtureLayer              */
#define LMC_MAX_MIX_ENTRIES 32    /* species over all MixtureLayers of one scene         */
#define LMC_MAX_SWEEP_SCENES 4096

typedef enum lmc_status {
  LMC_OK = 0,
  LMC_ERR_INVALID = 1,      /* bad scene / options (reference: std::invalid_argument) */
  LMC_ERR_CUDA = 2,         /* a CUDA runtime call failed                           */
  LMC_ERR_NOMEM = 3,        /* device or host allocation failed                     */
  LMC_ERR_KERNEL = 4,       /* the kernel raised its device error word              */
  LMC_ERR_UNSUPPORTED = 5   /* valid for the reference but outside this library     */
} lmc_status;

/* How a medium's phase function turns a uniform u into theta
 * (PhaseFunction::sample_theta, src/phase.cpp:78-304). */
typedef enum lmc_theta_kind {
  LMC_THETA_TABLE = 0,      /* inverse-CDF table over theta (RD, RD-EMC, Mie)        */
  LMC_THETA_TABLE_COS = 1,  /* inverse-CDF table over cos(theta) (Rayleigh, Draine)  */
  LMC_THETA_HG = 2,         /* Henyey-Greenstein closed form                         */
  LMC_THETA_UNIFORM = 3     /* acos(2u - 1)                                          */
} lmc_theta_kind;

/* One scattering medium (ScatteringMedium + its PhaseFunction,
 * include/luminis/core/medium.hpp:71-345).  Tables are host arrays copied by
 * lmc_create; the caller may free them afterwards. */
typedef struct lmc_medium_desc {
  int theta_kind;               /* lmc_theta_kind                                      */
  double hg_g;                  /* LMC_THETA_HG                                        */
  int theta_n;                  /* SamplingTable nodes (nDiv + 1)                      */
  const double *theta_values;   /* SamplingTable::values (src/table.cpp:27-31)         */
  const double *theta_cdf;      /* SamplingTable::cdf    (src/table.cpp:38-47)         */
  int amp_n;                    /* DataTable nodes, uniform in theta from 0            */
  double amp_dtheta;            /* DataTable spacing (pi / (amp_n - 1))                */
  const double *amp_s1;         /* S1(theta_i), interleaved re, im (amp_n complex)     */
  const double *amp_s2;         /* S2(theta_i), interleaved re, im                     */
  double mu_a, mu_s;            /* 1/mm; mu_t = mu_a + mu_s (src/medium.cpp:61-71)     */
  double mean_free_path;        /* mm; free paths are -mfp*ln(u) (src/medium.cpp:123)  */
  double cross_section;         /* mm^2; single-particle scattering cross-section
                                   Q_sca pi r^2 of the phase function
                                   (include/luminis/core/medium.hpp:186-188); read for
                                   MixtureLayer species only; <= 0: none              */
} lmc_medium_desc;

/* One slab z in [z_min, z_max): a HomogeneousLayer of `medium`
 * (include/luminis/core/sample.hpp:120-147), or a MixtureLayer (sample.hpp:150-205,
 * src/sample.cpp:41-104) of n_species co-located media at number densities n_i:
 * mu_s_i = n_i sigma_s_i, mu_a = sum mu_s_i (mu_a/mu_s)_i, free paths with the mean
 * 1 / sum mu_s_i, and one uniform per vertex selects the species by mu_s_i. */
typedef struct lmc_layer_desc {
  double z_min, z_max;          /* z_max may be +inf for the last layer                */
  int medium;                   /* HomogeneousLayer: index into media[]                */
  int n_species;                /* 0: HomogeneousLayer; 1..LMC_MAX_SPECIES: MixtureLayer */
  int species[LMC_MAX_SPECIES]; /* MixtureLayer: media[] indices of the species        */
  double number_density[LMC_MAX_SPECIES];  /* MixtureLayer: n_i, 1/mm^3                */
} lmc_layer_desc;

/* Laser (include/luminis/core/laser.hpp:24-96). */
typedef struct lmc_laser_desc {
  double position[3], direction[3], local_m[3], local_n[3];
  double jones[4];              /* m.re, m.im, n.re, n.im                              */
  double wavelength;            /* vacuum wavelength; photon k = 2 pi / wavelength     */
  double sigma;
  int source;                   /* 0 Point, 1 Uniform disk, 2 Gaussian                 */
  int temporal;                 /* 0 Delta, 1 Gaussian, 2 TopHat, 3 Exponential,
                                   4 PulseTrain, 5 CW                                  */
  double pulse_duration, repetition_rate, time_offset;
} lmc_laser_desc;

typedef enum lmc_sensor_kind {
  LMC_SENSOR_FARFIELD_CBS = 0,      /* FarFieldCBSSensor (src/detector.cpp:851-1310)  */
  LMC_SENSOR_PLANAR_FLUENCE = 1,    /* PlanarFluenceSensor (src/detector.cpp:704-841) */
  LMC_SENSOR_PLANAR_FIELD = 2,      /* PlanarFieldSensor (src/detector.cpp:490-568)   */
  LMC_SENSOR_FARFIELD_FLUENCE = 3,  /* far-field |E_f|^2 Stokes on (theta, phi); no
                                       counterpart in the reference's sources         */
  LMC_SENSOR_STATISTICS = 4         /* StatisticsSensor (src/detector.cpp:1569-1888)  */
} lmc_sensor_kind;

/* StatisticsSensor histograms (include/luminis/core/detector.hpp:595-699): counts of
 * the crossings a sensor takes, each histogram present when its bit of `set` is:
 *  events [0, n_events); theta = acos(-s_z) on [theta_min, theta_max) in n_theta bins;
 *  phi = atan2(s_y, s_x) in [0, 2 pi) on [phi_min, phi_max); penetration depth on
 *  [0, depth_max); arrival time t on bins [1, n_time) of width time_max / n_time;
 *  weight on [0, weight_max).  The first four have the sensor's time axis (len_t, dt:
 *  slice 0 integrated, slice floor(t/dt)+1 the window), time and weight do not. */
enum { LMC_STAT_EVENTS = 1, LMC_STAT_THETA = 2, LMC_STAT_PHI = 4, LMC_STAT_DEPTH = 8,
       LMC_STAT_TIME = 16, LMC_STAT_WEIGHT = 32 };
typedef struct lmc_statistics_desc {
  int set;
  int n_events;
  int n_theta; double theta_min, theta_max;
  int n_phi; double phi_min, phi_max;
  int n_depth; double depth_max;
  int n_time; double time_max;
  int n_weight; double weight_max;
} lmc_statistics_desc;

/* One sensor (Sensor + subclass fields, include/luminis/core/detector.hpp:95-562).
 * Filters follow Sensor::check_conditions (src/detector.cpp:374-417). */
typedef struct lmc_sensor_desc {
  int kind;
  double z;
  int absorb, estimator;
  int f_theta; double theta_min, theta_max;
  int f_phi; double phi_min, phi_max;
  int f_pos; double x_min, x_max, y_min, y_max;
  int f_dir; int direction;         /* 0 Forward, 1 Backward, 2 Both                  */
  int f_events; int events_min, events_max;
  double len_x, len_y, len_t, dx, dy, dt;              /* planar sensors            */
  double theta_max_grid, phi_max_grid, dtheta, dphi;   /* far-field sensors         */
  double theta_pp_max;          /* estimator-mode FarFieldCBS: theta cap of the estimated
                                   grid, <= 0 none (FarFieldCBSSensor::theta_pp_max)   */
  lmc_statistics_desc stats;    /* LMC_SENSOR_STATISTICS                               */
} lmc_sensor_desc;

/* Absorption recorder (include/luminis/core/absortion.hpp:34-80,
 * src/absortion.cpp:13-91): every scattering event deposits w mu_a/mu_t of the
 * layer (1 where the layer has mu_t = 0) at the photon's position, binned on a
 * cylindrical grid of n_r = floor(radius/d_r)+1 by n_z = floor(depth/d_z)+1 cells
 * (r = sqrt(x^2+y^2) <= radius, 0 <= z <= depth).  d_t > 0 adds time slices:
 * n_t = ceil(t_max/d_t)+1, slice 0 time-integrated and slice floor(t/d_t)+1 the
 * window of arrival time t = launch time + path length. */
typedef struct lmc_absorption_desc {
  int enabled;
  double radius, depth, d_r, d_z;
  double d_t, t_max;            /* d_t = 0: time-integrated only                     */
} lmc_absorption_desc;

/* Tally-layout slot of the Absorption grid: [n_t][n_r][n_z], dims {n_t, n_r, n_z, 1},
 * stored after the sensors. */
#define LMC_TALLY_ABSORPTION (-2)

/* The scene: Sample + Laser + SensorsGroup of a SimConfig
 * (include/luminis/core/simulation.hpp:67-90). */
typedef struct lmc_scene {
  double n_host;                /* Sample(n_medium): light_speed = 1 / n_host          */
  int n_media;
  lmc_medium_desc media[LMC_MAX_MEDIA];
  int n_layers;
  lmc_layer_desc layers[LMC_MAX_LAYERS];
  lmc_laser_desc laser;
  int n_sensors;
  lmc_sensor_desc sensors[LMC_MAX_SENSORS];
  lmc_absorption_desc absorption;   /* SimConfig::absorption (NULL: enabled = 0)     */
} lmc_scene;

typedef enum lmc_precision {
  LMC_PRECISION_FP32 = 0,       /* fp32 transport, fp64 CBS phase, fp64 tallies        */
  LMC_PRECISION_FP64 = 1        /* fp64 throughout (strict per-photon replay)          */
} lmc_precision;

/* How the hit-queue tally kernel adds hits into the direct-hit sensor grids
 * (lmc_run_opts.tally_mode).  The reference adds into per-thread sensor copies merged
 * after the run (src/simulation.cpp:131-139, 229-236); on the GPU every mode gives the same sums
 * up to the order of binary64 additions. */
typedef enum lmc_tally_mode {
  LMC_TALLY_DEFAULT = 0,        /* the library's choice: LMC_TALLY_GLOBAL                */
  LMC_TALLY_GLOBAL = 1,         /* one global atomic add per Stokes value per hit          */
  LMC_TALLY_WARP = 2,           /* lanes of a warp adding into the same grid cell combine
                                   their values first (match + shuffles): one global
                                   atomic per distinct cell and Stokes value               */
  LMC_TALLY_SHARED = 3          /* every block of the tally kernel keeps a private copy of
                                   the PlanarFluence / FarFieldCBS / FarFieldFluence grids
                                   that fit in its shared memory (smallest first), adds
                                   into it with shared atomics and adds it into the
                                   tallies once at its end; the other grids as GLOBAL.
                                   Single-scene handles only (a sweep: LMC_ERR_INVALID)  */
} lmc_tally_mode;

typedef struct lmc_run_opts {
  int precision;                /* lmc_precision                                       */
  int max_events;               /* SimConfig::MAX_EVENTS                               */
  int track_reverse_paths;      /* SimConfig::track_reverse_paths                      */
  int block_size;               /* 0: default                                          */
  int blocks_per_sm;            /* 0: as many as fit                                   */
  void *records;                /* optional device array of n_photons lmc_record       */
  void *stream;                 /* cudaStream_t to launch on; NULL: the handle's own   */
  uint64_t batch_photons;       /* photons per transport batch (hit-queue mode); 0: 32 Mi */
  int stream_format;            /* 0: u24 for FP32, u53 for FP64; 1: u24 for both (an FP64
                                   run on the FP32 run's numbers: precision alone)      */
  int host_tallies_zero;        /* lmc_run_host only: the caller's host tallies are all zero,
                                   so the device copy is cleared instead of uploaded     */
  int cbs_phase;                /* FarFieldCBS geometric phase k (s_out + s_in).(r_n - r_1):
                                   0 in binary64 (default), 1 in binary32 (precision study) */
  int stage_tables;             /* binary32 transport: copy every medium's amplitude table
                                   into each block's shared memory (1-D bulk copies) when
                                   that keeps the blocks per SM; 0 reads them through L1  */
  int no_replay;                /* 1: the transport keeps every photon's reverse-path history
                                   instead of replaying the photons a FarFieldCBS grid reads
                                   (replay is used by queued runs without records or
                                   estimator sensors, likelihood-ratio runs included)     */
  int tally_mode;               /* lmc_tally_mode of the hit-queue tally kernel (queued
                                   runs; inline runs add with global atomics)             */
} lmc_run_opts;

/* Final state of one photon, written when opts.records is set (the same layout as
 * the oracle's per-photon record). */
typedef struct lmc_record {
  uint64_t photon;
  uint32_t events, draws;
  int32_t fate, layer;          /* fate: 1 detected, 2 escaped, 3 left the stack at an
                                   interface, 4 roulette, 5 event cap                  */
  double weight, opticalpath, penetration_depth, launch_time;
  double pos[3], dir[3], m[3], n[3];
  double E[4];
  double r1[3], rn[3];
  double Er[4];
  double hit[3];
  int32_t n_hits, pad;
} lmc_record;

typedef struct lmc_stats {
  uint64_t photons, events, steps, detected, escaped, stack, roulette, cap, draws;
  uint64_t hits[LMC_MAX_SENSORS];   /* Sensor::hits increments                         */
  uint32_t error_flags;             /* device error word (0 = none)                    */
  float kernel_ms;                  /* whole run on the device (all launches), CUDA events */
  float transport_ms;               /* sum of the transport kernel launches alone       */
  uint32_t transport_launches;      /* transport kernel launches (queue batches)        */
  uint32_t replay_launches;         /* CBS replay kernel launches (0: no replay)        */
  uint64_t replayed;                /* photons whose reverse path the replay rebuilt    */
} lmc_stats;

typedef struct lmc_handle lmc_handle;

/* Validate a scene, upload its tables and allocate the handle's device scratch.
 * Replaces the set-up half of run_simulation_parallel (validate_sim_config,
 * per-thread sensor clones; src/simulation.cpp:95-143). */
LMC_API lmc_status lmc_create(const lmc_scene *scene, lmc_handle **out);

/* Release everything lmc_create allocated. */
LMC_API void lmc_destroy(lmc_handle *h);

/* Tally layout of sensor `sensor` inside the handle's tally buffer (doubles).
 * sensor = -1 returns the total size in *count; LMC_TALLY_ABSORPTION the Absorption
 * grid (count 0 without one).  dims as in the oracle:
 *  FARFIELD_CBS [8][N_t][N_theta][N_phi], PLANAR_FLUENCE [4][N_t][N_x][N_y],
 *  PLANAR_FIELD [2][N_x][N_y][2], FARFIELD_FLUENCE [4][N_t][N_theta][N_phi],
 *  STATISTICS counts (as doubles) of the histograms present, one after another:
 *  events [N_t][n_events], theta [N_t][n_theta], phi [N_t][n_phi], depth
 *  [N_t][n_depth], time [n_time], weight [n_weight]; dims {N_t, count, 0, 0}. */
LMC_API lmc_status lmc_tally_layout(const lmc_handle *h, int sensor, size_t *offset, size_t *count,
                            int dims[4]);

/* Transport photons [photon_begin, photon_begin + n_photons) under `seed` and ADD
 * their contributions into the device tally buffer d_tallies (size from
 * lmc_tally_layout(-1)).  Replaces the worker loop and merge of
 * run_simulation_parallel (src/simulation.cpp:157-243) and run_photon
 * (src/simulation.cpp:255-617).  Asynchronous on the handle's stream except for
 * the statistics read-back when `stats` is non-NULL. */
LMC_API lmc_status lmc_run(lmc_handle *h, uint64_t seed, uint64_t photon_begin, uint64_t n_photons,
                   const lmc_run_opts *opts, double *d_tallies, lmc_stats *stats);

/* lmc_run with HOST tallies: copies h_tallies to the device, runs, and copies the
 * sum back (the whole call is synchronous).  This is the path a reference-side
 * binding uses when it owns plain host arrays. */
LMC_API lmc_status lmc_run_host(lmc_handle *h, uint64_t seed, uint64_t photon_begin, uint64_t n_photons,
                        const lmc_run_opts *opts, double *h_tallies, lmc_stats *stats);

/* Copy of the last error message on this thread; returns its length. */
LMC_API size_t lmc_last_error(char *buf, size_t len);

/* lmc_create + lmc_run + lmc_destroy in one call that allocates no memory: for
 * callers that cannot allocate device memory, e.g. a host program that runs inside
 * a memory pool it does not own, or one that must not let cudaMalloc's implicit
 * device synchronisation stall other streams.  `scene` holds HOST pointers (as for
 * lmc_create); d_tallies is caller-owned device memory sized as lmc_tally_layout
 * reports for the same scene, and contributions are ADDED to it.  Everything else
 * (device scene, derived tables, run counters, hit queue) lives in one static
 * 64 MiB device array that the CUDA runtime reserves per GPU when this library is
 * loaded.  Limits: the scene's tables must fit in 8 MiB (a larger scene returns
 * LMC_ERR_INVALID with the size it needs); photons are processed in batches that
 * fit the remaining ~56 MiB hit queue, or of opts->batch_photons when that is
 * smaller.  opts->block_size and opts->blocks_per_sm pick the launch shape and the
 * kernel variant, and opts->tally_mode the tally kernel's mode, as they do for lmc_run
 * (LMC_TALLY_SHARED's private grids are the kernel's shared memory, not an allocation).  The first call on each device looks up the
 * array's device address (cudaGetSymbolAddress), so make that first call before
 * any stream capture.  All calls on one device share the array: calls that
 * overlap in time -- from two threads, or on two streams -- race and corrupt each
 * other's results; serialise them.  Runs on opts->stream (NULL = legacy default
 * stream) and is synchronous: it copies the run counters back and returns only
 * after the stream has finished the run.  stats->kernel_ms is
 * always 0 (timing events would be allocations).
 * No counterpart in the reference. */
LMC_API lmc_status lmc_run_noalloc(const lmc_scene *scene, uint64_t seed, uint64_t photon_begin,
                                   uint64_t n_photons, const lmc_run_opts *opts, double *d_tallies,
                                   lmc_stats *stats);

/* ---- sweeps: many independent scenes in one launch ------------------------------------ */
/* A parameter sweep of the reference is a sequence of run_simulation_parallel calls, one
 * per scene (src/simulation.cpp:105-249).  A sweep handle transports all of them in one
 * persistent launch: photons are numbered across the scenes in order, scene s owning
 * [P_s, P_s + n_s) with P_s = n_0 + ... + n_{s-1}, and photon g draws the stream of
 * (seed, g).  Scene s's tallies therefore equal those of lmc_run(seed, P_s, n_s) on a
 * handle of that scene alone.  Every scene must put every sensor plane at z <= 0. */
LMC_API lmc_status lmc_create_sweep(const lmc_scene *scenes, int n_scenes, lmc_handle **out);

/* Sensor `sensor` of scene `scene` in the sweep's tally buffer (scene = -1: total size in
 * *count; sensor = LMC_TALLY_ABSORPTION: the scene's Absorption grid); dims as
 * lmc_tally_layout. */
LMC_API lmc_status lmc_sweep_layout(const lmc_handle *h, int scene, int sensor, size_t *offset,
                                    size_t *count, int dims[4]);

/* Photons per scene for the following lmc_run_sweep calls (n_scenes counts; synchronous:
 * set them before capturing lmc_run_sweep in a CUDA graph). */
LMC_API lmc_status lmc_sweep_set_photons(lmc_handle *h, const uint64_t *n_photons);

/* Transport every scene's photons and ADD their contributions into d_tallies (size from
 * lmc_sweep_layout(-1)).  With stats == NULL the call only enqueues work on opts->stream
 * (no host synchronisation, no allocation once the hit queue has grown): it can be
 * captured in a CUDA graph after one uncaptured call of the same size. */
LMC_API lmc_status lmc_run_sweep(lmc_handle *h, uint64_t seed, const lmc_run_opts *opts,
                                 double *d_tallies, lmc_stats *stats);

/* Launch shape picked by lmc_autotune. */
typedef struct lmc_tune_result {
  int block_size;               /* threads per block                                   */
  int blocks_per_sm;            /* 0: as many as fit                                   */
  uint64_t batch_photons;       /* photons per hit-queue batch                         */
  double photons_per_s;         /* the shape's rate on the sample (device time)        */
  uint64_t sample_photons;      /* photons of the sample                               */
  int n_tried;
  int tally_mode;               /* lmc_tally_mode picked (queued runs; else the options') */
} lmc_tune_result;

/* Times candidate launch shapes -- threads per block (256, 128), resident blocks per SM
 * (as many as fit, 2, 1: the persistent grid, hence photons per thread) and photons per
 * hit-queue batch (32 Mi, 8 Mi) -- on a sample of about sample_photons photons (a
 * sweep: every scene's count scaled down, restored afterwards) with the rest of `opts`;
 * then, at the fastest shape, the tally modes (LMC_TALLY_GLOBAL, _WARP and, for a
 * single scene, _SHARED) of hit-queue runs.  Returns the fastest; copy its fields into
 * lmc_run_opts for the real runs.  Runs into a scratch tally buffer (allocates it);
 * synchronous. */
LMC_API lmc_status lmc_autotune(lmc_handle *h, uint64_t seed, const lmc_run_opts *opts,
                                uint64_t sample_photons, lmc_tune_result *out);

/* Sensor hit counts of the last lmc_run_sweep, [n_scenes][LMC_MAX_SENSORS] (synchronises). */
LMC_API lmc_status lmc_sweep_hits(lmc_handle *h, uint64_t *hits);

/* ---- likelihood-ratio derivatives ("adjoint") --------------------------------------- */
/* Derivatives of selected outputs with respect to every medium's parameters
 * (mu_a, mu_s, mean_free_path, HG g), K = 4 n_media, estimated in the same transport
 * pass by the likelihood-ratio (score) method: every hit contributes v * (1, s_1..s_K),
 * s = d log(path density x weight) / d param accumulated over the photon's flights,
 * albedo factors and HG angle draws.  Running per-photon sums; no path is stored.
 * No counterpart in the reference (config "Differentiable" of the task). */
typedef struct lmc_adjoint_opts {
  int radial_sensor;           /* PlanarFluenceSensor: total S0 of its time-integrated
                                  grid + radial S0 profile by hit radius; -1: none    */
  int radial_bins;             /* 1..512                                              */
  double radial_max;           /* profile covers r in [0, radial_max)                 */
} lmc_adjoint_opts;

/* Outputs per row (n_out doubles): [total, radial_bins bins] when radial_sensor >= 0,
 * then for each FarFieldCBSSensor S0 coherent and S0 incoherent, [N_t][N_theta][N_phi]
 * each.  The buffer holds (1 + n_params) rows: the outputs, then d outputs / d param k
 * for k = 4 medium + (0 mu_a, 1 mu_s, 2 mean_free_path, 3 g).  Needs every sensor plane
 * at z <= 0 and at most 4 media. */
LMC_API lmc_status lmc_adjoint_layout(const lmc_handle *h, const lmc_adjoint_opts *a, size_t *n_out,
                                      int *n_params);

/* lmc_run that also ADDS the outputs and their derivatives into d_adjoint (device,
 * (1 + n_params) x n_out doubles). */
LMC_API lmc_status lmc_run_adjoint(lmc_handle *h, uint64_t seed, uint64_t photon_begin,
                                   uint64_t n_photons, const lmc_run_opts *opts,
                                   const lmc_adjoint_opts *a, double *d_tallies, double *d_adjoint,
                                   lmc_stats *stats);

/* Likelihood-ratio outputs of a sweep (lmc_create_sweep): scene s has its own block of
 * (1 + n_params_s) rows of n_out_s doubles (layout as lmc_adjoint_layout for that scene,
 * n_params_s = 4 x its media) at *offset in the sweep's adjoint buffer; scene = -1
 * returns the buffer's total size in *n_out and the largest n_params.  One set of options
 * for every scene (radial_sensor >= 0 must name a PlanarFluenceSensor in each). */
LMC_API lmc_status lmc_sweep_adjoint_layout(const lmc_handle *h, const lmc_adjoint_opts *a, int scene,
                                            size_t *offset, size_t *n_out, int *n_params);

/* lmc_run_sweep that also ADDS every scene's outputs and derivatives into its block of
 * d_adjoint (device, size from lmc_sweep_adjoint_layout(-1)).  Scene s's block equals
 * lmc_run_adjoint on a handle of that scene alone over photons [P_s, P_s + n_s).  The
 * first run with a set of options uploads the per-scene layouts synchronously; later
 * runs with the same options enqueue device work only (graph-capturable). */
LMC_API lmc_status lmc_run_sweep_adjoint(lmc_handle *h, uint64_t seed, const lmc_run_opts *opts,
                                         const lmc_adjoint_opts *a, double *d_tallies,
                                         double *d_adjoint, lmc_stats *stats);

/* Backward pass: d_grad_params[k] = sum_j d_adjoint[(1 + k) n_out + j] * d_grad_out[j]
 * (all device pointers; enqueued on `stream`, NULL = legacy default stream). */
LMC_API lmc_status lmc_adjoint_contract(const double *d_adjoint, const double *d_grad_out,
                                        size_t n_out, int n_params, double *d_grad_params,
                                        void *stream);

/* ---- set-up physics (host), the constructors' work -------------------------------- */

/* Mie amplitudes S1, S2 (interleaved re/im) at the n cosines mu for size parameter x
 * and relative index m; efficiencies and g.  Replaces miev/mievinfo
 * (src/mie/dmiev.cpp:45-76, src/mie/MIEV0noP.f). */
LMC_API lmc_status lmc_mie(double x, double m_re, double m_im, int n, const double *mu, double *s1,
                   double *s2, double *qext, double *qsca, double *g);

typedef enum lmc_pdf_kind {
  LMC_PDF_RAYLEIGH = 1, LMC_PDF_RD = 3, LMC_PDF_RDEMC = 4, LMC_PDF_DRAINE = 5, LMC_PDF_MIE = 6
} lmc_pdf_kind;

/* Phase-function parameters for lmc_sampling_table / lmc_phase_cross_section. */
typedef struct lmc_phase_params {
  int kind;                     /* lmc_pdf_kind                                        */
  double g, a;                  /* Draine                                              */
  double wavelength, radius, n_particle, n_medium;
} lmc_phase_params;

/* SamplingTable of a tabulated phase function: values and cdf (n_div + 1 each).
 * Replaces SamplingTable::initialize with the phase functions' PDFs
 * (src/table.cpp:6-48, src/phase.cpp:87-304). */
LMC_API lmc_status lmc_sampling_table(const lmc_phase_params *p, int n_div, double min_val,
                              double max_val, double *values, double *cdf);

/* Single-particle scattering cross-section sigma_s (RD-EMC, Mie;
 * src/phase.cpp:168-200, :270-284). */
LMC_API lmc_status lmc_phase_cross_section(const lmc_phase_params *p, double *sigma_s);

typedef enum lmc_amp_kind { LMC_AMP_RGD = 0, LMC_AMP_MIE = 1 } lmc_amp_kind;

/* Amplitude tables S1(theta_i), S2(theta_i), theta_i = i*pi/(n-1): RGDMedium uses
 * n = 2000 (src/medium.cpp:77-120), MieMedium n = 1000 with x = 2 pi r / lambda
 * (src/medium.cpp:160-236). */
LMC_API lmc_status lmc_amplitude_table(int kind, double radius, double n_particle, double n_medium,
                               double wavelength, int n, double *s1, double *s2);

/* One Mie species of a batched table build: MiePhaseFunction(wavelength, radius,
 * n_particle, n_medium, ...) with MieMedium(phase, radius, n_particle, n_medium, wavelength). */
typedef struct lmc_mie_species {
  double wavelength, radius, n_particle, n_medium;
} lmc_mie_species;

/* The set-up tables of n Mie species built together on the current CUDA device, bit for bit
 * the numbers the per-species calls give:
 *   values[n_div + 1]          sampling nodes min_val + i (max_val - min_val) / n_div (shared)
 *   cdf[n][n_div + 1]          lmc_sampling_table(LMC_PDF_MIE, n_div, min_val, max_val)
 *   sigma[n]                   lmc_phase_cross_section(LMC_PDF_MIE)
 *   s1[n][2 n_amp], s2[...]    lmc_amplitude_table(LMC_AMP_MIE, n_amp), interleaved re/im
 * All are host arrays.  values/cdf/sigma may be null together (n_div ignored), s1/s2 may be
 * null together or n_amp 0 (no amplitude tables).  The Mie coefficient recurrence runs on
 * the host; the angular sums, the PDF and the CDF on the GPU.  timing_ms (4 doubles, may
 * be null) receives the host series, upload, device-kernel and read-back times in ms.
 * Replaces the per-species
 * construction of MiePhaseFunction (src/phase.cpp:244-304, src/table.cpp:6-48) and
 * MieMedium (src/medium.cpp:160-236) around MIEV0 (src/mie/MIEV0noP.f). */
LMC_API lmc_status lmc_mie_tables(const lmc_mie_species *species, int n, int n_div,
                                  double min_val, double max_val, int n_amp, double *values,
                                  double *cdf, double *sigma, double *s1, double *s2,
                                  double *timing_ms);

/* ---- measurement --------------------------------------------------------------------- */

/* Measured FP32 FMA issue rate of the current GPU (TFLOP/s, 2 flops per FMA): the
 * roofline denominator of the transport kernel, which is FP32/SFU-issue bound.
 * No counterpart in the reference (it has no GPU code). */
LMC_API lmc_status lmc_probe_fp32_peak(int iters, double *tflops, double *ms);

#ifdef __cplusplus
}
#endif
#endif
