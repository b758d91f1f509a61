"""luminis_mc_b200 -- B200 (sm_100a) drop-in for luminis-mc's photon propagation.

``import luminis_mc_b200 as luminis_mc`` gives the reference's scene API
(phase functions, media, Sample, Laser, sensors, SimConfig) and a
``run_simulation_parallel`` that runs the transport as one CUDA kernel through
the C ABI of include/luminis_b200.h.  ``postprocess_*`` normalise the tallies as
the reference does.
"""
from .core import (Absorption, CMatrix, CrossingDirection, CVec2, DrainePhaseFunction,  # noqa: F401
                   FarFieldCBSSensor, FarFieldFluenceSensor, HenyeyGreensteinPhaseFunction, Laser,
                   LaserSource, Layer, LogLevel, Matrix, MiePhaseFunction, MieMedium, MixtureLayer,
                   mie_species,
                   PhaseFunction, PhotonRecordSensor, PlanarFieldSensor, PlanarFluenceSensor,
                   RayleighDebyeEMCPhaseFunction, RayleighDebyePhaseFunction,
                   RayleighPhaseFunction, RGDMedium, Rng, Sample, SampleLayer, ScatteringMedium,
                   Sensor, SensorsGroup, StatisticsSensor, TemporalProfile,
                   UniformPhaseFunction, Vec2, Vec3, calculate_rotation_angle, cross, dot,
                   form_factor, gaussian_distribution, matcmul, matcmulscalar, norm,
                   set_log_level, solid_angle_bin, uniform_distribution)
from .simulation import (FarFieldCBSProcessed, PlanarFieldProcessed,  # noqa: F401
                         PlanarFluenceProcessed, SimConfig, StokesMatrixProcessed, Transport,
                         last_run_stats, postprocess_farfield_cbs, postprocess_farfield_fluence,
                         postprocess_planar_field, postprocess_planar_fluence,
                         release_gpu_cache, run_simulation_parallel, validate_sim_config)

# enum values exported at module level, as pybind's export_values() does
Point, Uniform, Gaussian = LaserSource.Point, LaserSource.Uniform, LaserSource.Gaussian
Forward, Backward, Both = (CrossingDirection.Forward, CrossingDirection.Backward,
                           CrossingDirection.Both)
Delta, TopHat, ExponentialTime, PulseTrain, CW = (
    TemporalProfile.Delta, TemporalProfile.TopHat, TemporalProfile.ExponentialTime,
    TemporalProfile.PulseTrain, TemporalProfile.CW)
