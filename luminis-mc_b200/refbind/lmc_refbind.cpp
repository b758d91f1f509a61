// lmc_refbind.cpp -- the reference's own Python objects on the GPU.
//
// A pybind11 module (_lmc_refbind) whose run_simulation_parallel(config) takes the
// SimConfig a user built with the reference's Python API (luminis_mc._core,
// python/python_module.cpp:114-673), reads its Sample, Laser, SensorsGroup and
// Absorption, runs the photon transport on the GPU through this library's C ABI
// (include/luminis_b200.h: lmc_create, lmc_run_host, lmc_destroy) and ADDS the
// tallies and hit counts into the reference's own sensor arrays, as the reference's
// run_simulation_parallel merges its thread-local clones into them
// (src/simulation.cpp:233-243).  The reference's postprocess_* then run unchanged on
// those arrays (src/results.cpp:5-101).
//
// Built against the reference's headers only; no object of the reference is linked,
// so the module works beside whatever build of luminis_mc._core the user imported
// (it shares that module's pybind11 type registry):
//   * a layer, medium, phase function or sensor is identified by the name of its
//     dynamic type (typeid of the object, demangled), which reads the object's own
//     vtable and needs no type-information symbol of the reference's library;
//   * the members the reference keeps private -- each table-based phase function's
//     SamplingTable and the Henyey-Greenstein g (include/luminis/sample/phase.hpp:
//     77-189) -- are read through member pointers taken in explicit template
//     instantiations, the one place where C++ does not check access
//     ([temp.spec.general]).  The GPU therefore samples exactly the tables the
//     reference built, with no recomputation;
//   * the amplitude tables are the media's public DataTables S1_table / S2_table
//     (include/luminis/core/medium.hpp:223-224, :286-287).
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cxxabi.h>

#include <array>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <typeinfo>
#include <vector>

#include <luminis/core/simulation.hpp>
#include <luminis/sample/phase.hpp>
#include <luminis/sample/table.hpp>

#include "luminis_b200.h"

namespace py = pybind11;
using namespace luminis::core;
using luminis::math::CMatrix;
using luminis::math::Matrix;
namespace ls = luminis::sample;

namespace {

// ------------------------------------------------------------- private members
// Expose<Tag, &Class::member> defines member(Tag) returning the member pointer; the
// explicit instantiations below name private members, which is allowed there.
template <typename Tag, typename Tag::type M> struct Expose {
  friend typename Tag::type member(Tag) { return M; }
};

#define LMC_PRIVATE(TAG, CLASS, TYPE, NAME)                                                 \
  struct TAG {                                                                              \
    using type = TYPE CLASS::*;                                                             \
    friend type member(TAG);                                                                \
  };                                                                                        \
  template struct Expose<TAG, &CLASS::NAME>;

LMC_PRIVATE(RayleighTable, ls::RayleighPhaseFunction, ls::SamplingTable, table)
LMC_PRIVATE(RdTable, ls::RayleighDebyePhaseFunction, ls::SamplingTable, table)
LMC_PRIVATE(RdemcTable, ls::RayleighDebyeEMCPhaseFunction, ls::SamplingTable, table)
LMC_PRIVATE(DraineTable, ls::DrainePhaseFunction, ls::SamplingTable, table)
LMC_PRIVATE(MieTable, ls::MiePhaseFunction, ls::SamplingTable, table)
LMC_PRIVATE(HgG, ls::HenyeyGreensteinPhaseFunction, double, g)
#undef LMC_PRIVATE

// ------------------------------------------------------------------- helpers
// Qualified name of an object's dynamic type, e.g. "luminis::sample::MiePhaseFunction".
template <typename T> std::string dynamic_name(const T &obj)
{
  const char *mangled = typeid(obj).name();
  int status = 0;
  char *d = abi::__cxa_demangle(mangled, nullptr, nullptr, &status);
  std::string out = (status == 0 && d) ? d : mangled;
  std::free(d);
  return out;
}

[[noreturn]] void not_supported(const std::string &what)
{
  PyErr_SetString(PyExc_NotImplementedError, what.c_str());
  throw py::error_already_set();
}

void check(lmc_status s)
{
  if (s == LMC_OK)
    return;
  char msg[1024];
  lmc_last_error(msg, sizeof msg);
  if (s == LMC_ERR_INVALID)
    throw std::invalid_argument(msg);                     // ValueError, as the reference
  if (s == LMC_ERR_UNSUPPORTED)
    not_supported(msg);
  throw std::runtime_error(msg);
}

struct HandleGuard {
  lmc_handle *h = nullptr;
  ~HandleGuard() { lmc_destroy(h); }
};

// Host arrays a scene points into, alive until lmc_create has copied them.
struct Keep {
  std::vector<std::vector<double>> arrays;
  const double *add(std::vector<double> v)
  {
    arrays.push_back(std::move(v));
    return arrays.back().data();
  }
};

std::vector<double> interleave(const std::vector<std::complex<double>> &y)
{
  std::vector<double> out(2 * y.size());
  for (size_t i = 0; i < y.size(); ++i) {
    out[2 * i] = y[i].real();
    out[2 * i + 1] = y[i].imag();
  }
  return out;
}

// ------------------------------------------------------------- scene from objects
// One medium: coefficients (ScatteringMedium, include/luminis/core/medium.hpp:71-190),
// mean free path and amplitude tables of the RGD / Mie medium, theta sampler of its
// phase function.
void medium_desc(const ScatteringMedium &m, lmc_medium_desc &d, Keep &keep)
{
  std::memset(&d, 0, sizeof d);
  const std::string mk = dynamic_name(m);
  const ls::DataTable *s1 = nullptr, *s2 = nullptr;
  if (mk == "luminis::core::MieMedium") {
    const auto &mm = static_cast<const MieMedium &>(m);
    d.mean_free_path = mm.mean_free_path;
    s1 = &mm.S1_table;
    s2 = &mm.S2_table;
  } else if (mk == "luminis::core::RGDMedium") {
    const auto &rm = static_cast<const RGDMedium &>(m);
    d.mean_free_path = rm.mean_free_path;
    s1 = &rm.S1_table;
    s2 = &rm.S2_table;
  } else {
    not_supported("medium " + mk + " has no GPU transport");
  }
  if (!s1->uniform_ || !s2->uniform_ || s1->y_values.size() != s2->y_values.size() ||
      s1->dx_ != s2->dx_ || s1->x_min_ != 0.0 || s2->x_min_ != 0.0)
    not_supported("amplitude tables on a non-uniform theta grid");
  d.amp_n = (int)s1->y_values.size();
  d.amp_dtheta = s1->dx_;
  d.amp_s1 = keep.add(interleave(s1->y_values));
  d.amp_s2 = keep.add(interleave(s2->y_values));
  d.mu_a = m.mu_absorption;
  d.mu_s = m.mu_scattering;

  const ls::PhaseFunction *ph = m.phase_function;
  if (!ph)
    throw std::invalid_argument("ScatteringMedium: Phase function is not defined!");
  const std::string pk = dynamic_name(*ph);
  // sigma_s from the two phase functions that define one (src/phase.cpp:168-186,
  // :270-282); the base class's version ends the process, so it is never called
  if (pk == "luminis::sample::MiePhaseFunction" || pk == "luminis::sample::RayleighDebyeEMCPhaseFunction")
    d.cross_section = ph->scattering_cross_section();
  const ls::SamplingTable *t = nullptr;
  d.theta_kind = LMC_THETA_TABLE;
  if (pk == "luminis::sample::HenyeyGreensteinPhaseFunction") {
    d.theta_kind = LMC_THETA_HG;
    d.hg_g = static_cast<const ls::HenyeyGreensteinPhaseFunction &>(*ph).*member(HgG{});
  } else if (pk == "luminis::sample::UniformPhaseFunction") {
    d.theta_kind = LMC_THETA_UNIFORM;
  } else if (pk == "luminis::sample::MiePhaseFunction") {
    t = &(static_cast<const ls::MiePhaseFunction &>(*ph).*member(MieTable{}));
  } else if (pk == "luminis::sample::RayleighDebyeEMCPhaseFunction") {
    t = &(static_cast<const ls::RayleighDebyeEMCPhaseFunction &>(*ph).*member(RdemcTable{}));
  } else if (pk == "luminis::sample::RayleighDebyePhaseFunction") {
    t = &(static_cast<const ls::RayleighDebyePhaseFunction &>(*ph).*member(RdTable{}));
  } else if (pk == "luminis::sample::RayleighPhaseFunction") {
    d.theta_kind = LMC_THETA_TABLE_COS;                   // its table is over cos(theta)
    t = &(static_cast<const ls::RayleighPhaseFunction &>(*ph).*member(RayleighTable{}));
  } else if (pk == "luminis::sample::DrainePhaseFunction") {
    d.theta_kind = LMC_THETA_TABLE_COS;
    t = &(static_cast<const ls::DrainePhaseFunction &>(*ph).*member(DraineTable{}));
  } else {
    not_supported("phase function " + pk + " has no GPU sampler");
  }
  if (t) {
    if (t->values.size() != t->cdf.size() || t->values.empty())
      throw std::invalid_argument("phase function sampling table is empty");
    d.theta_n = (int)t->values.size();
    d.theta_values = keep.add(t->values);
    d.theta_cdf = keep.add(t->cdf);
  }
}

void vec3(double *dst, const luminis::math::Vec3 &v)
{
  dst[0] = v.x;
  dst[1] = v.y;
  dst[2] = v.z;
}

// Sensor filters (Sensor, include/luminis/core/detector.hpp:95-160) and the geometry of
// each kind.
void sensor_desc(const Sensor &s, lmc_sensor_desc &d)
{
  std::memset(&d, 0, sizeof d);
  d.z = s.origin.z;
  d.absorb = s.absorb_photons;
  d.estimator = s.estimator_enabled;
  d.f_theta = s.filter_theta_enabled;
  d.theta_min = s.filter_theta_min;
  d.theta_max = s.filter_theta_max;
  d.f_phi = s.filter_phi_enabled;
  d.phi_min = s.filter_phi_min;
  d.phi_max = s.filter_phi_max;
  d.f_pos = s.filter_position_enabled;
  d.x_min = s.filter_x_min;
  d.x_max = s.filter_x_max;
  d.y_min = s.filter_y_min;
  d.y_max = s.filter_y_max;
  d.f_dir = s.filter_direction_enabled;
  d.direction = (int)s.filter_direction;
  d.f_events = s.filter_events_enabled;
  d.events_min = s.filter_events_min;
  d.events_max = s.filter_events_max;
  const std::string k = dynamic_name(s);
  if (k == "luminis::core::FarFieldCBSSensor") {
    const auto &f = static_cast<const FarFieldCBSSensor &>(s);
    d.kind = LMC_SENSOR_FARFIELD_CBS;
    d.theta_max_grid = f.theta_max;
    d.phi_max_grid = f.phi_max;
    d.dtheta = f.dtheta;
    d.dphi = f.dphi;
    d.len_t = f.t_max;
    d.dt = f.dt;
    d.theta_pp_max = f.theta_pp_max;
    if (f.phi_explicit) {
      if (f.estimator_enabled)
        not_supported("estimator-mode FarFieldCBSSensor with explicit phi slices");
      d.phi_max_grid = f.N_phi * f.dphi;                  // the slices set the column count
    }
  } else if (k == "luminis::core::PlanarFluenceSensor") {
    const auto &p = static_cast<const PlanarFluenceSensor &>(s);
    d.kind = LMC_SENSOR_PLANAR_FLUENCE;
    d.len_x = p.len_x;
    d.len_y = p.len_y;
    d.len_t = p.len_t;
    d.dx = p.dx;
    d.dy = p.dy;
    d.dt = p.dt;
  } else if (k == "luminis::core::PlanarFieldSensor") {
    const auto &p = static_cast<const PlanarFieldSensor &>(s);
    d.kind = LMC_SENSOR_PLANAR_FIELD;
    d.len_x = p.len_x;
    d.len_y = p.len_y;
    d.dx = p.dx;
    d.dy = p.dy;
  } else if (k == "luminis::core::StatisticsSensor") {
    const auto &q = static_cast<const StatisticsSensor &>(s);
    d.kind = LMC_SENSOR_STATISTICS;
    d.len_t = q.t_max;
    d.dt = q.dt;
    lmc_statistics_desc &h = d.stats;
    h.set = (q.events_histogram_bins_set ? LMC_STAT_EVENTS : 0) |
            (q.theta_histogram_bins_set ? LMC_STAT_THETA : 0) |
            (q.phi_histogram_bins_set ? LMC_STAT_PHI : 0) |
            (q.depth_histogram_bins_set ? LMC_STAT_DEPTH : 0) |
            (q.time_histogram_bins_set ? LMC_STAT_TIME : 0) |
            (q.weight_histogram_bins_set ? LMC_STAT_WEIGHT : 0);
    h.n_events = q.max_events;
    h.n_theta = q.n_bins_theta;
    h.theta_min = q.min_theta;
    h.theta_max = q.max_theta;
    h.n_phi = q.n_bins_phi;
    h.phi_min = q.min_phi;
    h.phi_max = q.max_phi;
    h.n_depth = q.n_bins_depth;
    h.depth_max = q.max_depth;
    h.n_time = q.time_histogram_bins_set ? (int)q.time_histogram.size() : 0;
    h.time_max = q.h_max_time;
    h.n_weight = q.n_bins_weight;
    h.weight_max = q.max_weight;
  } else {
    not_supported(k + " is not supported by the GPU transport");
  }
}

// ------------------------------------------------------------ tallies into objects
void add_matrix(Matrix &m, const double *src, size_t n)
{
  if ((size_t)m.rows * m.cols != n)
    throw std::runtime_error("tally layout does not match the sensor's grid");
  double *dst = m.data.data();
  for (size_t i = 0; i < n; ++i)
    dst[i] += src[i];
}

void add_grids(std::vector<Matrix> &grids, const double *src, size_t cell)
{
  for (size_t t = 0; t < grids.size(); ++t)
    add_matrix(grids[t], src + t * cell, cell);
}

void add_counts(std::vector<int> &h, const double *src)
{
  for (size_t i = 0; i < h.size(); ++i)
    h[i] += (int)std::llround(src[i]);
}

// Sensor i's slice of the flat tallies, in the layout lmc_tally_layout reports (the
// reference's own array order), added into the sensor object.
void add_sensor(Sensor &s, const lmc_sensor_desc &d, const double *src, const int dims[4])
{
  if (d.kind == LMC_SENSOR_FARFIELD_CBS) {
    auto &f = static_cast<FarFieldCBSSensor &>(s);
    const size_t cell = (size_t)dims[2] * dims[3], plane = (size_t)dims[1] * cell;
    std::vector<Matrix> *g[8] = {&f.S0_coh, &f.S1_coh, &f.S2_coh, &f.S3_coh,
                                 &f.S0_incoh, &f.S1_incoh, &f.S2_incoh, &f.S3_incoh};
    for (int q = 0; q < 8; ++q)
      add_grids(*g[q], src + q * plane, cell);
  } else if (d.kind == LMC_SENSOR_PLANAR_FLUENCE) {
    auto &p = static_cast<PlanarFluenceSensor &>(s);
    const size_t cell = (size_t)dims[2] * dims[3], plane = (size_t)dims[1] * cell;
    std::vector<Matrix> *g[4] = {&p.S0, &p.S1, &p.S2, &p.S3};
    for (int q = 0; q < 4; ++q)
      add_grids(*g[q], src + q * plane, cell);
  } else if (d.kind == LMC_SENSOR_PLANAR_FIELD) {
    auto &p = static_cast<PlanarFieldSensor &>(s);
    const size_t n = (size_t)dims[1] * dims[2];
    CMatrix *g[2] = {&p.Ex, &p.Ey};
    for (int q = 0; q < 2; ++q) {
      if ((size_t)g[q]->rows * g[q]->cols != n)
        throw std::runtime_error("tally layout does not match the sensor's grid");
      std::complex<double> *dst = g[q]->data.data();
      const double *a = src + q * 2 * n;
      for (size_t i = 0; i < n; ++i)
        dst[i] += std::complex<double>(a[2 * i], a[2 * i + 1]);
    }
  } else if (d.kind == LMC_SENSOR_STATISTICS) {
    auto &q = static_cast<StatisticsSensor &>(s);
    const double *p = src;
    auto per_slice = [&](std::vector<std::vector<int>> &h) {
      for (auto &row : h) {
        add_counts(row, p);
        p += row.size();
      }
    };
    if (q.events_histogram_bins_set) per_slice(q.events_histogram);
    if (q.theta_histogram_bins_set) per_slice(q.theta_histogram);
    if (q.phi_histogram_bins_set) per_slice(q.phi_histogram);
    if (q.depth_histogram_bins_set) per_slice(q.depth_histogram);
    if (q.time_histogram_bins_set) {
      add_counts(q.time_histogram, p);
      p += q.time_histogram.size();
    }
    if (q.weight_histogram_bins_set) {
      add_counts(q.weight_histogram, p);
      p += q.weight_histogram.size();
    }
    if ((size_t)(p - src) != (size_t)dims[1])       // dims {N_t, count, 0, 0}
      throw std::runtime_error("tally layout does not match the statistics histograms");
  }
}

// ------------------------------------------------------------------- the scene
// The C scene of a SimConfig (include/luminis/core/simulation.hpp:67-90): the same
// validation errors as validate_sim_config (src/simulation.cpp:95-103), one medium
// descriptor per distinct ScatteringMedium, layers, laser, sensors, absorption.
void fill_scene(const SimConfig &config, lmc_scene &sc, Keep &keep)
{
  if (config.sample == nullptr)
    throw std::invalid_argument("SimConfig::sample must not be null");
  if (config.laser == nullptr)
    throw std::invalid_argument("SimConfig::laser must not be null");
  if (config.detector == nullptr)
    throw std::invalid_argument("SimConfig::detector must not be null");
  std::memset(&sc, 0, sizeof sc);
  const Sample &sample = *config.sample;
  sc.n_host = sample.refractive_index;
  if (sample.layers.size() > LMC_MAX_LAYERS)
    throw std::invalid_argument("at most " + std::to_string(LMC_MAX_LAYERS) + " layers");
  std::vector<const ScatteringMedium *> media;
  auto medium_index = [&](const ScatteringMedium *m) {
    for (size_t k = 0; k < media.size(); ++k)
      if (media[k] == m)
        return (int)k;
    if (media.size() == LMC_MAX_MEDIA)
      throw std::invalid_argument("at most " + std::to_string(LMC_MAX_MEDIA) + " distinct media");
    medium_desc(*m, sc.media[media.size()], keep);
    media.push_back(m);
    return (int)media.size() - 1;
  };
  for (size_t i = 0; i < sample.layers.size(); ++i) {
    const Layer &L = *sample.layers[i];
    lmc_layer_desc &d = sc.layers[i];
    d.z_min = L.z_min;
    d.z_max = L.z_max;
    const std::string k = dynamic_name(L);
    if (k == "luminis::core::HomogeneousLayer") {
      d.medium = medium_index(static_cast<const HomogeneousLayer &>(L).medium);
    } else if (k == "luminis::core::MixtureLayer") {
      const auto &mx = static_cast<const MixtureLayer &>(L);
      if (mx.species.size() > LMC_MAX_SPECIES)
        not_supported("a MixtureLayer of more than " + std::to_string(LMC_MAX_SPECIES) + " species");
      d.medium = -1;
      d.n_species = (int)mx.species.size();
      for (size_t j = 0; j < mx.species.size(); ++j) {
        d.species[j] = medium_index(mx.species[j]);
        d.number_density[j] = mx.number_densities[j];
      }
    } else {
      not_supported("layer " + k + " has no GPU transport");
    }
  }
  sc.n_layers = (int)sample.layers.size();
  sc.n_media = (int)media.size();

  const Laser &las = *config.laser;                         // include/luminis/core/laser.hpp:24-96
  vec3(sc.laser.position, las.position);
  vec3(sc.laser.direction, las.direction);
  vec3(sc.laser.local_m, las.local_m);
  vec3(sc.laser.local_n, las.local_n);
  sc.laser.jones[0] = las.polarization.m.real();
  sc.laser.jones[1] = las.polarization.m.imag();
  sc.laser.jones[2] = las.polarization.n.real();
  sc.laser.jones[3] = las.polarization.n.imag();
  sc.laser.wavelength = las.wavelength;
  sc.laser.sigma = las.sigma;
  sc.laser.source = (int)las.source_type;
  sc.laser.temporal = (int)las.temporal_profile;
  sc.laser.pulse_duration = las.pulse_duration;
  sc.laser.repetition_rate = las.repetition_rate;
  sc.laser.time_offset = las.time_offset;

  const SensorsGroup &group = *config.detector;
  if (group.detectors.size() > LMC_MAX_SENSORS)
    throw std::invalid_argument("at most " + std::to_string(LMC_MAX_SENSORS) + " sensors");
  for (size_t i = 0; i < group.detectors.size(); ++i)
    sensor_desc(*group.detectors[i], sc.sensors[i]);
  sc.n_sensors = (int)group.detectors.size();
  if (config.absorption) {                                  // include/luminis/core/absortion.hpp:34-80
    const Absorption &a = *config.absorption;
    sc.absorption.enabled = 1;
    sc.absorption.radius = a.radius;
    sc.absorption.depth = a.depth;
    sc.absorption.d_r = a.d_r;
    sc.absorption.d_z = a.d_z;
    sc.absorption.d_t = a.d_t;
    sc.absorption.t_max = a.t_max;
  }
}

// The scene as the GPU receives it, for inspection: the lmc_scene bytes with every
// table pointer cleared, and per medium its (theta values, theta cdf, S1, S2) tables.
py::tuple describe(const SimConfig &config)
{
  lmc_scene sc;
  Keep keep;
  fill_scene(config, sc, keep);
  py::list tables;
  for (int i = 0; i < sc.n_media; ++i) {
    lmc_medium_desc &m = sc.media[i];
    auto arr = [](const double *p, size_t n) { return py::bytes(reinterpret_cast<const char *>(p), n * 8); };
    tables.append(py::make_tuple(arr(m.theta_values, m.theta_n), arr(m.theta_cdf, m.theta_n),
                                 arr(m.amp_s1, 2 * (size_t)m.amp_n), arr(m.amp_s2, 2 * (size_t)m.amp_n)));
    m.theta_values = m.theta_cdf = m.amp_s1 = m.amp_s2 = nullptr;
  }
  return py::make_tuple(py::bytes(reinterpret_cast<const char *>(&sc), sizeof sc), tables);
}

// ---------------------------------------------------------------------- the run
// run_simulation_parallel(config) with the photons transported on the GPU: the
// tallies of photons [0, n_photons) under config.seed added into config.detector's
// sensors and config.absorption, each sensor's hits incremented.  n_threads,
// batch_size, pin_threads_to_cores and show_progress have no meaning here and are
// ignored.
py::dict run(SimConfig &config, const std::string &precision)
{
  if (precision != "fp32" && precision != "fp64")
    throw std::invalid_argument("precision must be 'fp32' or 'fp64'");
  lmc_scene sc;
  Keep keep;
  fill_scene(config, sc, keep);
  SensorsGroup &group = *config.detector;

  lmc_run_opts o;
  std::memset(&o, 0, sizeof o);
  o.precision = precision == "fp64" ? LMC_PRECISION_FP64 : LMC_PRECISION_FP32;
  o.max_events = config.MAX_EVENTS;
  o.track_reverse_paths = config.track_reverse_paths ? 1 : 0;
  o.host_tallies_zero = 1;
  lmc_stats st;
  std::memset(&st, 0, sizeof st);
  std::vector<double> flat;
  std::vector<size_t> off(sc.n_sensors);
  std::vector<std::array<int, 4>> dims(sc.n_sensors);
  size_t abs_off = 0, abs_count = 0;
  int abs_dims[4] = {0, 0, 0, 0};
  {
    py::gil_scoped_release release;                         // as the reference's binding does
    HandleGuard g;
    check(lmc_create(&sc, &g.h));
    size_t total = 0;
    check(lmc_tally_layout(g.h, -1, nullptr, &total, nullptr));
    for (int i = 0; i < sc.n_sensors; ++i) {
      size_t cnt = 0;
      check(lmc_tally_layout(g.h, i, &off[i], &cnt, dims[i].data()));
    }
    check(lmc_tally_layout(g.h, LMC_TALLY_ABSORPTION, &abs_off, &abs_count, abs_dims));
    flat.assign(total, 0.0);
    check(lmc_run_host(g.h, config.seed, 0, config.n_photons, &o, flat.data(), &st));
  }
  for (int i = 0; i < sc.n_sensors; ++i) {
    add_sensor(*group.detectors[i], sc.sensors[i], flat.data() + off[i], dims[i].data());
    group.detectors[i]->hits += st.hits[i];
  }
  if (config.absorption && abs_count)
    add_grids(config.absorption->time_slices, flat.data() + abs_off, (size_t)abs_dims[1] * abs_dims[2]);

  py::dict out;
  out["photons"] = st.photons;
  out["events"] = st.events;
  out["steps"] = st.steps;
  out["detected"] = st.detected;
  out["escaped"] = st.escaped;
  out["kernel_ms"] = st.kernel_ms;
  return out;
}

}  // namespace

PYBIND11_MODULE(_lmc_refbind, m)
{
  m.doc() = "run_simulation_parallel on the GPU for the reference's own SimConfig objects";
  m.def("run_simulation_parallel", &run, py::arg("config"), py::arg("precision") = "fp32",
        "Transport config.n_photons photons on the GPU and add every sensor's tallies and hits "
        "into the reference's own objects (the reference's run_simulation_parallel contract); "
        "returns the run's counters");
  m.def("describe", &describe, py::arg("config"),
        "The scene the GPU receives for this config: (lmc_scene bytes with table pointers "
        "cleared, [(theta values, theta cdf, S1, S2) per medium] as float64 bytes)");
}
