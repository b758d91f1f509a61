/*
 * oracle/lmc_oracle.h -- TEST INFRASTRUCTURE (the oracle).  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 *
 * Plain-C restatement of the reference's photon-propagation path:
 * run_simulation_parallel + run_photon (src/simulation.cpp:105-617), the
 * sensor dispatch SensorsGroup::record_hit (src/detector.cpp:178-270), the
 * direct-hit sensors (FarFieldCBS, PlanarFluence, PlanarField) with the CBS
 * reverse path (src/detector.cpp:490-1310), the source (src/laser.cpp), the
 * layered sample (src/sample.cpp), media and phase functions
 * (src/medium.cpp, src/phase.cpp) and their tables (src/table.cpp).
 *
 * The scene is described by the same physical parameters the reference's
 * constructors take, and the oracle builds its own tables from them (Mie via
 * oracle/miev0.c), so table construction is checked as well as transport.
 *
 * Random streams: the reference's own xoshiro256++ per-photon seeding
 * (src/rng.cpp, include/luminis/math/rng.hpp) or the Philox replay stream of
 * oracle/philox_ref.h in either format.
 */
#ifndef LMC_ORACLE_H
#define LMC_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LMC_O_MAX_PHASE 16
#define LMC_O_MAX_MEDIA 16
#define LMC_O_MAX_LAYERS 16
#define LMC_O_MAX_SENSORS 8
#define LMC_O_MAX_SPECIES 8

enum lmc_o_phase_kind {
  LMC_O_PHASE_UNIFORM = 0,    /* src/phase.cpp:78-83   */
  LMC_O_PHASE_RAYLEIGH = 1,   /* src/phase.cpp:87-98   */
  LMC_O_PHASE_HG = 2,         /* src/phase.cpp:102-115 */
  LMC_O_PHASE_RD = 3,         /* src/phase.cpp:119-142 */
  LMC_O_PHASE_RDEMC = 4,      /* src/phase.cpp:146-214 */
  LMC_O_PHASE_DRAINE = 5,     /* src/phase.cpp:218-240 */
  LMC_O_PHASE_MIE = 6         /* src/phase.cpp:244-304 */
};

enum lmc_o_medium_kind { LMC_O_MEDIUM_RGD = 0, LMC_O_MEDIUM_MIE = 1 };

enum lmc_o_sensor_kind {
  LMC_O_SENSOR_FARFIELD_CBS = 0,
  LMC_O_SENSOR_PLANAR_FLUENCE = 1,
  LMC_O_SENSOR_PLANAR_FIELD = 2,
  LMC_O_SENSOR_FARFIELD_FLUENCE = 3,
  LMC_O_SENSOR_STATISTICS = 4      /* src/detector.cpp:1569-1888 */
};

/* StatisticsSensor histograms (include/luminis/core/detector.hpp:595-699), each
 * present when its bit of `set` is: 1 events [0, n_events), 2 theta, 4 phi,
 * 8 penetration depth, 16 arrival time, 32 weight.  The time resolution is the
 * sensor's len_t / dt (set_time_resolution). */
enum { LMC_O_STAT_EVENTS = 1, LMC_O_STAT_THETA = 2, LMC_O_STAT_PHI = 4, LMC_O_STAT_DEPTH = 8,
       LMC_O_STAT_TIME = 16, LMC_O_STAT_WEIGHT = 32 };
typedef struct lmc_o_statistics {
  int set;
  int n_events;
  int n_theta; double theta_min, theta_max;
  int n_phi; double phi_min, phi_max;
  int n_depth; double depth_max;
  int n_time; double time_max;
  int n_weight; double weight_max;
} lmc_o_statistics;

enum lmc_o_rng { LMC_O_RNG_XOSHIRO = 0, LMC_O_RNG_PHILOX_U53 = 1, LMC_O_RNG_PHILOX_U24 = 2 };

enum lmc_o_fate {
  LMC_O_FATE_DETECTED = 1,   /* killed by an absorbing sensor            */
  LMC_O_FATE_ESCAPED = 2,    /* left the sample (is_inside false)        */
  LMC_O_FATE_STACK = 3,      /* left the stack during interface crossing */
  LMC_O_FATE_ROULETTE = 4,
  LMC_O_FATE_EVENT_CAP = 5
};

typedef struct lmc_o_phase {
  int kind;
  double g, a;                            /* HG g; Draine g, a          */
  double wavelength, radius, n_particle, n_medium;
  int n_div;
  double min_val, max_val;
} lmc_o_phase;

typedef struct lmc_o_medium {
  int kind;                               /* lmc_o_medium_kind          */
  int phase;                              /* index into scene.phase     */
  double radius, n_particle, n_medium, wavelength;
  double mu_a, mu_s, mfp;
} lmc_o_medium;

/* HomogeneousLayer of `medium` (n_species == 0), or a MixtureLayer
 * (include/luminis/core/sample.hpp:150-205) of n_species co-located media at
 * number densities n_i [1/mm^3]: mu_s_i = n_i sigma_s_i with sigma_s_i the
 * species' phase-function scattering cross-section (Mie and RD-EMC only). */
typedef struct lmc_o_layer {
  int medium;
  double z_min, z_max;
  int n_species;
  int species[LMC_O_MAX_SPECIES];
  double number_density[LMC_O_MAX_SPECIES];
} lmc_o_layer;

typedef struct lmc_o_laser {
  double position[3], direction[3], local_m[3], local_n[3];
  double pol[4];                          /* m.re, m.im, n.re, n.im     */
  double wavelength, sigma;
  int source;                             /* 0 Point, 1 Uniform, 2 Gaussian */
  int temporal;                           /* 0 Delta .. 5 CW            */
  double pulse_duration, repetition_rate, time_offset;
} lmc_o_laser;

typedef struct lmc_o_sensor {
  int kind;
  double z;
  int absorb, estimator;
  /* filters (src/detector.cpp:374-417) */
  int f_theta; double theta_min, theta_max;
  int f_phi; double phi_min, phi_max;
  int f_pos; double x_min, x_max, y_min, y_max;
  int f_dir; int direction;               /* 0 Forward, 1 Backward, 2 Both */
  int f_events; int events_min, events_max;
  /* planar sensors */
  double len_x, len_y, len_t, dx, dy, dt;
  /* far-field sensors (len_t and dt above are the time axis) */
  double theta_max_grid, phi_max_grid, dtheta, dphi;
  double theta_pp_max;                    /* estimator: theta cap of the grid (0: none) */
  lmc_o_statistics stats;                 /* STATISTICS sensors                        */
} lmc_o_sensor;

/* Absorption recorder (include/luminis/core/absortion.hpp:34-80): the weight each
 * event deposits, binned on a cylindrical (r, z) grid of n_r = floor(radius/d_r)+1 by
 * n_z = floor(depth/d_z)+1 cells; with d_t > 0 also by time, n_t = ceil(t_max/d_t)+1
 * slices with slice 0 time-integrated. */
typedef struct lmc_o_absorption {
  int enabled;
  double radius, depth, d_r, d_z, d_t, t_max;
} lmc_o_absorption;

typedef struct lmc_o_scene {
  double n_host;
  int n_phase; lmc_o_phase phase[LMC_O_MAX_PHASE];
  int n_media; lmc_o_medium media[LMC_O_MAX_MEDIA];
  int n_layers; lmc_o_layer layers[LMC_O_MAX_LAYERS];
  lmc_o_laser laser;
  int n_sensors; lmc_o_sensor sensors[LMC_O_MAX_SENSORS];
  lmc_o_absorption absorption;
} lmc_o_scene;

/* Final state of one photon (per-photon replay comparison). */
typedef struct lmc_o_record {
  uint64_t photon;
  uint32_t events, draws;
  int32_t fate, layer;
  double weight, opticalpath, penetration_depth, launch_time;
  double pos[3], dir[3], m[3], n[3];
  double E[4];                            /* forward Jones (m.re, m.im, n.re, n.im) */
  double r1[3], rn[3];
  double Er[4];                           /* reverse Jones at CBS detection, else 0 */
  double hit[3];                          /* last sensor hit point, else 0          */
  int32_t n_hits, pad;
} lmc_o_record;

typedef struct lmc_o_stats {
  uint64_t photons, events, steps, detected, escaped, stack, roulette, cap, draws;
} lmc_o_stats;

typedef struct lmc_o_handle lmc_o_handle;

lmc_o_handle *lmc_oracle_create(const lmc_o_scene *scene, char *err, int err_len);
void lmc_oracle_destroy(lmc_o_handle *h);

/* Doubles a sensor's tally occupies and its shape.  Sensor index n_sensors is the
 * Absorption grid when the scene has one: [n_t][n_r][n_z], dims {n_t, n_r, n_z, 1}.
 * Layouts:
 *  FARFIELD_CBS      [8 stokes: S0..S3 coherent, S0..S3 incoherent][N_t][N_theta][N_phi]
 *  PLANAR_FLUENCE    [4][N_t][N_x][N_y]
 *  PLANAR_FIELD      [2: Ex, Ey][N_x][N_y][2: re, im]
 *  FARFIELD_FLUENCE  [4][N_t][N_theta][N_phi]
 *  STATISTICS        counts, the histograms present one after another:
 *                    events [N_t][n_events], theta [N_t][n_theta], phi [N_t][n_phi],
 *                    depth [N_t][n_depth], time [n_time], weight [n_weight];
 *                    dims {N_t, n_doubles, 0, 0}                                  */
int lmc_oracle_sensor_shape(const lmc_o_handle *h, int sensor, int dims[4], size_t *n_doubles);

/* Photons [begin, begin+count) with seed; tallies[s] accumulate (caller zeroes),
 * tallies[n_sensors] the Absorption grid when the scene has one;
 * records (optional) gets count entries; hits[s] incremented. */
int lmc_oracle_run(lmc_o_handle *h, uint64_t seed, uint64_t begin, uint64_t count, int rng,
                   int max_events, int track_reverse, double **tallies, uint64_t *hits,
                   lmc_o_record *records, lmc_o_stats *stats);

/* Likelihood-ratio derivatives of selected outputs with respect to each medium's
 * parameters, in the order (mu_a, mu_s, mean_free_path, HG g) per medium:
 * K = 4 n_media.  Outputs (n_out doubles per row):
 *   [radial sensor]   total S0 of the PlanarFluence sensor's time-integrated grid,
 *                     then radial_bins bins of the same S0 by hit radius
 *                     sqrt(x^2+y^2) < radial_max                (if radial_sensor >= 0)
 *   [each FarFieldCBS] S0 coherent then S0 incoherent, [N_t][N_theta][N_phi] each
 * out has (1 + K) rows: row 0 the outputs, row 1 + k their derivative for param k.
 * The estimator: every hit contributes v * (1, s_1..s_K), s = the photon's score,
 * the derivative of log(path density x weight) accumulated over its history:
 * free flights (exponential with mean mean_free_path, crossings rescaled by the
 * mu_t ratio), albedo factors mu_s/mu_t and HG angle densities. */
typedef struct lmc_o_adjoint {
  int radial_sensor;
  int radial_bins;
  double radial_max;
} lmc_o_adjoint;

size_t lmc_oracle_adjoint_outputs(const lmc_o_handle *h, const lmc_o_adjoint *a);
int lmc_oracle_run_adjoint(lmc_o_handle *h, uint64_t seed, uint64_t begin, uint64_t count, int rng,
                           int max_events, int track_reverse, double **tallies, uint64_t *hits,
                           const lmc_o_adjoint *a, double *out, lmc_o_stats *stats);

/* Tables the oracle built (for table parity): theta sampling table of a medium's
 * phase function (values/cdf of n_div+1), and amplitude tables (n complex). */
int lmc_oracle_phase_table(const lmc_o_handle *h, int medium, int *n, const double **values,
                           const double **cdf);
int lmc_oracle_amp_table(const lmc_o_handle *h, int medium, int *n, double *dtheta,
                         const double **s1, const double **s2);
double lmc_oracle_phase_sample_theta(const lmc_o_handle *h, int medium, double u);

/* The Philox4x32-10 block function and the stream contract (oracle/philox_ref.h). */
void lmc_oracle_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double lmc_oracle_stream_uniform(uint64_t seed, uint64_t photon, uint64_t draw, int format);

/* MIEV0 restatement helpers (oracle/miev0.c). */
int lmc_oracle_miev0_selftest(double *worst_rel_err);
void lmc_oracle_mie(double x, double m_re, double m_im, int n, const double *mu, double *s1,
                    double *s2, double *qext, double *qsca, double *g);

#ifdef __cplusplus
}
#endif
#endif
