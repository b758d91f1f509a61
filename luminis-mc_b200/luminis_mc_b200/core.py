"""Scene objects with the luminis-mc Python API (python/python_module.cpp:27-662).

Same class names, constructor arguments, attributes and error behaviour as the
reference's pybind module, so scripts written for ``luminis_mc`` build their
scene unchanged.  Tables are built at construction by the native library
(lmc_sampling_table, lmc_amplitude_table, lmc_mie), and sensor tallies are
float64 numpy arrays whose per-time-bin ``Matrix`` views are what the
reference exposes as ``std::vector<Matrix>``.
"""
from __future__ import annotations

import copy
import enum
import math
import random

import numpy as np

from . import _native as N

# ----------------------------------------------------------------------------- math
class Vec3:
    """3-vector (include/luminis/math/vec.hpp:48-80)."""
    __slots__ = ("x", "y", "z")

    def __init__(self, x: float = 0.0, y: float = 0.0, z: float = 0.0):
        self.x, self.y, self.z = float(x), float(y), float(z)

    def __iter__(self):
        return iter((self.x, self.y, self.z))

    def __repr__(self):
        return f"Vec3({self.x:.6f}, {self.y:.6f}, {self.z:.6f})"


class Vec2:
    __slots__ = ("x", "y")

    def __init__(self, x: float = 0.0, y: float = 0.0):
        self.x, self.y = float(x), float(y)


class CVec2:
    """Jones vector (m, n) (include/luminis/math/vec.hpp:94-101)."""
    __slots__ = ("m", "n")

    def __init__(self, m: complex = 0j, n: complex = 0j):
        self.m, self.n = complex(m), complex(n)


class Matrix(np.ndarray):
    """Row-major float64 matrix; a numpy array, so the buffer protocol works as in
    the reference (python/python_module.cpp:65-86)."""

    def __new__(cls, rows: int, cols: int):
        return np.zeros((int(rows), int(cols)), dtype=np.float64).view(cls)

    @property
    def rows(self):
        return self.shape[0]

    @property
    def cols(self):
        return self.shape[1]

    def get(self, i, j):
        return float(self[i, j])

    def set(self, i, j, value):
        self[i, j] = value

    def get_numpy(self):
        return np.asarray(self).copy()


class CMatrix(np.ndarray):
    """Row-major complex128 matrix (python/python_module.cpp:88-111)."""

    def __new__(cls, rows: int, cols: int):
        return np.zeros((int(rows), int(cols)), dtype=np.complex128).view(cls)

    @staticmethod
    def identity(size: int):
        m = CMatrix(size, size)
        for i in range(size):
            m[i, i] = 1.0
        return m

    @property
    def rows(self):
        return self.shape[0]

    @property
    def cols(self):
        return self.shape[1]

    def get(self, i, j):
        return complex(self[i, j])

    def set(self, i, j, value):
        self[i, j] = value

    def get_numpy(self):
        return np.asarray(self).copy()


def dot(a: Vec3, b: Vec3) -> float:
    return a.x * b.x + a.y * b.y + a.z * b.z


def norm(v: Vec3) -> float:
    return math.sqrt(dot(v, v))


def cross(a: Vec3, b: Vec3) -> Vec3:
    """Cross product, normalised when non-zero (src/vec.cpp:14-26)."""
    r = Vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x)
    n = norm(r)
    if n > 0.0:
        inv = 1.0 / n
        r = Vec3(r.x * inv, r.y * inv, r.z * inv)
    return r


def matcmul(A, B, C):
    C[...] = np.asarray(A) @ np.asarray(B)


def matcmulscalar(scalar, A):
    A *= scalar


def calculate_rotation_angle(n_from: Vec3, n_to: Vec3) -> float:
    nu, nv = norm(n_from), norm(n_to)
    if nu < 1e-12 or nv < 1e-12:
        return 0.0
    c = max(-1.0, min(1.0, dot(n_from, n_to) / (nu * nv)))
    return math.acos(c)


def solid_angle_bin(i_theta: int, dtheta: float, dphi: float) -> float:
    """Solid angle of polar bin i (src/utils.cpp:76-82)."""
    return dphi * (math.cos(i_theta * dtheta) - math.cos((i_theta + 1) * dtheta))


def form_factor(theta: float, k: float, radius: float) -> float:
    """Sphere form factor (src/phase.cpp:10-20)."""
    if abs(theta) == 0.0:
        return 1.0
    u = 2.0 * k * radius * math.sin(theta / 2.0)
    return 3 * (math.sin(u) - u * math.cos(u)) / u ** 3


# ------------------------------------------------------------------------------ rng
class Rng:
    """xoshiro256++ seeded by SplitMix64, the reference's host generator
    (include/luminis/math/rng.hpp:53-89).  Not used by the GPU transport, which
    draws per-photon Philox streams."""
    _M = (1 << 64) - 1

    def __init__(self, seed: int | None = None):
        if seed is None:
            seed = random.getrandbits(32)
        z = int(seed) & self._M
        self.s = []
        for _ in range(4):
            z = (z + 0x9E3779B97F4A7C15) & self._M
            x = z
            x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & self._M
            x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & self._M
            self.s.append(x ^ (x >> 31))

    def _next(self) -> int:
        s, M = self.s, self._M
        rotl = lambda x, k: ((x << k) | (x >> (64 - k))) & M
        result = (rotl((s[0] + s[3]) & M, 23) + s[0]) & M
        t = (s[1] << 17) & M
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t
        s[3] = rotl(s[3], 45)
        return result

    def uniform(self) -> float:
        return (self._next() >> 11) * 2.0 ** -53

    def normal(self, mean: float, stddev: float) -> float:
        u1 = self.uniform()
        while u1 <= 0.0:
            u1 = self.uniform()
        u2 = self.uniform()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2) * stddev + mean


# ------------------------------------------------------------------------------ enums
class _BoundEnum(enum.Enum):
    """An enumeration with the semantics of the reference's bound C++ enums (pybind11,
    python/python_module.cpp): members carry .name and .value, int() and operator.index
    give the value and the hash is the value's, but a member is not an int, does not
    compare equal to one and has no order.  Code that treats scalars and enums apart
    (the reference's HDF5 writer stores an enum by its name) sees the same types."""

    def __int__(self):
        return self.value

    def __index__(self):
        return self.value

    def __hash__(self):
        return hash(self.value)


class LaserSource(_BoundEnum):
    Point = 0
    Uniform = 1
    Gaussian = 2


class TemporalProfile(_BoundEnum):
    Delta = 0
    Gaussian = 1
    TopHat = 2
    ExponentialTime = 3
    PulseTrain = 4
    CW = 5


class CrossingDirection(_BoundEnum):
    Forward = 0
    Backward = 1
    Both = 2


class LogLevel(_BoundEnum):
    debug = 0
    info = 1
    warn = 2
    error = 3
    off = 4


_log_level = LogLevel.info


def set_log_level(level):
    global _log_level
    _log_level = LogLevel(level)


# ---------------------------------------------------------------------- phase functions
def _sampling_table(params: N.PhaseParams, n_div: int, min_val: float, max_val: float):
    if int(n_div) <= 0:
        raise ValueError("nDiv must be greater than 0")
    if not float(min_val) < float(max_val):
        raise ValueError("minVal must be less than maxVal")
    values = np.zeros(int(n_div) + 1)
    cdf = np.zeros(int(n_div) + 1)
    N.check(N.lib().lmc_sampling_table(params, int(n_div), float(min_val), float(max_val),
                                       N.as_dptr(values), N.as_dptr(cdf)))
    return values, cdf


def _mie_at(x: float, m: complex, mu: np.ndarray):
    mu = np.ascontiguousarray(mu, dtype=np.float64)
    n = mu.size
    s1 = np.zeros(2 * max(n, 1))
    s2 = np.zeros(2 * max(n, 1))
    qe, qs, g = (np.zeros(1) for _ in range(3))
    N.check(N.lib().lmc_mie(float(x), m.real, m.imag, n, N.as_dptr(mu), N.as_dptr(s1),
                            N.as_dptr(s2), N.as_dptr(qe), N.as_dptr(qs), N.as_dptr(g)))
    return (s1[: 2 * n].view(np.complex128), s2[: 2 * n].view(np.complex128),
            (float(qe[0]), float(qs[0]), float(g[0])))


class PhaseFunction:
    """Base class (include/luminis/sample/phase.hpp:28-60)."""
    _theta_kind = N.THETA_TABLE

    def sample(self, x: float) -> float:
        """cos(theta) for a uniform x (sample_cos)."""
        raise NotImplementedError

    def sample_theta(self, x: float) -> float:
        return math.acos(self.sample(x))

    def sample_phi(self, x: float) -> float:
        return 2.0 * math.pi * x

    def sample_phi_conditional(self, theta, S, E, k, rng) -> float:
        """Polarisation-conditional azimuth by rejection (src/phase.cpp:27-49)."""
        S = np.asarray(S)
        s2sq, s1sq = abs(S[0, 0]) ** 2, abs(S[1, 1]) ** 2
        e1sq, e2sq = abs(E.m) ** 2, abs(E.n) ** 2
        e12 = (E.m * E.n.conjugate()).real
        a = s2sq * e1sq + s1sq * e2sq
        b = s1sq * e1sq + s2sq * e2sq
        c = 2.0 * (s2sq - s1sq) * e12
        fmax = 0.5 * (a + b) + 0.5 * math.sqrt((a - b) ** 2 + c * c)
        while True:
            phi = 2.0 * math.pi * rng.uniform()
            cp, sp = math.cos(phi), math.sin(phi)
            F = a * cp * cp + b * sp * sp + c * cp * sp
            if rng.uniform() * fmax <= max(F, 0.0):
                return phi

    def scattering_efficiency(self) -> float:
        raise NotImplementedError("PhaseFunction::scattering_efficiency: Not implemented for this "
                                  "phase function.")

    def scattering_cross_section(self) -> float:
        raise NotImplementedError("PhaseFunction::scattering_cross_section: Not implemented for this"
                                  " phase function.")

    def get_anisotropy_factor(self, n_samples: int = 200000):
        rng = Rng()
        c = np.array([self.sample(rng.uniform()) for _ in range(int(n_samples))])
        g = float(c.mean())
        return [g, float(math.sqrt(max(float((c * c).mean()) - g * g, 0.0) / n_samples))]

    # table access used by the scene packer
    def _table(self):
        return None, None


class _TablePhase(PhaseFunction):
    _samples_theta = True

    def _build(self, params, n_div, min_val, max_val):
        self.nDiv, self.minVal, self.maxVal = int(n_div), float(min_val), float(max_val)
        self._params = params
        self._values, self._cdf = _sampling_table(params, n_div, min_val, max_val)

    def _table(self):
        return self._values, self._cdf

    def _inverse(self, u: float) -> float:
        idx = int(np.searchsorted(self._cdf, u, side="left"))   # std::lower_bound
        if idx == 0:
            return float(self._values[0])
        if idx >= self._values.size:
            return float(self._values[-1])
        c0, c1 = self._cdf[idx - 1], self._cdf[idx]
        v0, v1 = self._values[idx - 1], self._values[idx]
        return float(v0 + (u - c0) / (c1 - c0) * (v1 - v0))

    def sample(self, x):
        v = self._inverse(x)
        return math.cos(v) if self._samples_theta else v

    def sample_theta(self, x):
        v = self._inverse(x)
        return v if self._samples_theta else math.acos(v)


class UniformPhaseFunction(PhaseFunction):
    _theta_kind = N.THETA_UNIFORM

    def sample(self, x):
        return 2.0 * x - 1.0


class HenyeyGreensteinPhaseFunction(PhaseFunction):
    """Closed-form HG sampling (src/phase.cpp:102-115)."""
    _theta_kind = N.THETA_HG

    def __init__(self, g: float):
        self.g = float(g)

    def sample(self, x):
        g = self.g
        gg = g * g
        frac = (1.0 - gg) / (1.0 - g + 2.0 * g * x)
        return (1.0 + gg - frac * frac) / (2.0 * g)


class RayleighPhaseFunction(_TablePhase):
    _theta_kind = N.THETA_TABLE_COS
    _samples_theta = False

    def __init__(self, nDiv: int, minVal: float, maxVal: float):
        self._build(N.PhaseParams(kind=N.PDF_RAYLEIGH), nDiv, minVal, maxVal)

    def pdf(self, x):
        return 0.375 * (1.0 + x * x)


class RayleighDebyePhaseFunction(_TablePhase):
    def __init__(self, wavelength, radius, nDiv, minVal, maxVal):
        self.wavelength, self.radius = float(wavelength), float(radius)
        self.k = 2 * math.pi / self.wavelength
        self._build(N.PhaseParams(kind=N.PDF_RD, wavelength=wavelength, radius=radius),
                    nDiv, minVal, maxVal)

    def pdf(self, x):
        return (1.0 / (4.0 * math.pi)) * form_factor(x, self.k, self.radius) ** 2


class RayleighDebyeEMCPhaseFunction(_TablePhase):
    def __init__(self, wavelength, radius, n_particle, n_medium, nDiv, minVal, maxVal):
        self.wavelength, self.radius = float(wavelength), float(radius)
        self.n_particle, self.n_medium = float(n_particle), float(n_medium)
        self.k = 2 * math.pi * self.n_medium / self.wavelength
        p = N.PhaseParams(kind=N.PDF_RDEMC, wavelength=wavelength, radius=radius,
                          n_particle=n_particle, n_medium=n_medium)
        sig = np.zeros(1)
        N.check(N.lib().lmc_phase_cross_section(p, N.as_dptr(sig)))
        self._sigma = float(sig[0])
        self._build(p, nDiv, minVal, maxVal)

    def scattering_cross_section(self):
        return self._sigma

    def scattering_efficiency(self):
        return self._sigma / (math.pi * self.radius ** 2)

    def rho_phase_function(self, x):
        m1 = self.n_particle / self.n_medium - 1.0
        v = (4.0 / 3.0) * math.pi * self.radius ** 3
        F = form_factor(x, self.k, self.radius)
        return (self.k ** 4 / (4.0 * math.pi * self._sigma)) * m1 * m1 * v * v * F * F * (
            1.0 + math.cos(x) ** 2)

    def pdf(self, x):
        return self.rho_phase_function(x) * math.sin(x)


class DrainePhaseFunction(_TablePhase):
    _theta_kind = N.THETA_TABLE_COS
    _samples_theta = False

    def __init__(self, g, a, nDiv, minVal, maxVal):
        self.g, self.a = float(g), float(a)
        self._build(N.PhaseParams(kind=N.PDF_DRAINE, g=g, a=a), nDiv, minVal, maxVal)

    def pdf(self, x):
        g, a = self.g, self.a
        hg = (1.0 - g * g) / (1.0 + g * g - 2.0 * g * x) ** 1.5
        return (1.0 / 4.0 * math.pi) * hg * (1.0 + a * x * x) / (3 + a * (1 + 2 * g * g))


class MiePhaseFunction(_TablePhase):
    """Mie theta sampler; PDF from the Mie series with x = k r, k = 2 pi n_m / lambda
    (src/phase.cpp:244-304)."""

    def __init__(self, wavelength, radius, n_particle, n_medium, nDiv, minVal, maxVal):
        p = self._set_particle(wavelength, radius, n_particle, n_medium)
        sig = np.zeros(1)
        N.check(N.lib().lmc_phase_cross_section(p, N.as_dptr(sig)))
        self._sigma = float(sig[0])
        self._build(p, nDiv, minVal, maxVal)

    def _set_particle(self, wavelength, radius, n_particle, n_medium) -> N.PhaseParams:
        self.wavelength, self.radius = float(wavelength), float(radius)
        self.n_particle, self.n_medium = float(n_particle), float(n_medium)
        self.k = 2 * math.pi * self.n_medium / self.wavelength
        self.m = complex(self.n_particle / self.n_medium, 0.0)
        return N.PhaseParams(kind=N.PDF_MIE, wavelength=wavelength, radius=radius,
                             n_particle=n_particle, n_medium=n_medium)

    def scattering_cross_section(self):
        return self._sigma

    def scattering_efficiency(self):
        return self._sigma / (math.pi * self.radius ** 2)

    def rho_phase_function(self, x):
        mu = min(1.0, max(-1.0, math.cos(x)))
        s1, s2, _ = _mie_at(self.k * self.radius, self.m, np.array([mu]))
        return (math.pi / (self.k * self.k * self._sigma)) * (abs(s1[0]) ** 2 + abs(s2[0]) ** 2)

    def pdf(self, x):
        return self.rho_phase_function(x) * math.sin(x)


# ------------------------------------------------------------------------------- media
class ScatteringMedium:
    """Base class (include/luminis/core/medium.hpp:71-195)."""

    def __init__(self, phase_func: PhaseFunction):
        self.phase_function = phase_func
        self.mu_a = 0.0
        self.mu_s = 0.0
        self.mu_t = 0.0
        self.mean_free_path = 0.0

    def set_scattering_coefficient(self, mu_s):
        self.mu_s = float(mu_s)
        self.mu_t = self.mu_a + self.mu_s

    def set_absorption_coefficient(self, mu_a):
        self.mu_a = float(mu_a)
        self.mu_t = self.mu_a + self.mu_s

    def set_mean_free_path(self, mfp):
        """Mean free path of free-path sampling; does NOT update mu_s / mu_t."""
        self.mean_free_path = float(mfp)

    def sample_free_path(self, rng) -> float:
        return -1 * self.mean_free_path * math.log(rng.uniform())

    def sample_scattering_angle(self, rng) -> float:
        return self.phase_function.sample_theta(rng.uniform())

    def sample_azimuthal_angle(self, rng) -> float:
        return self.phase_function.sample_phi(rng.uniform())

    def sample_conditional_azimuthal_angle(self, rng, S, E, theta) -> float:
        return self.phase_function.sample_phi_conditional(theta, S, E, self.k, rng)

    def scattering_matrix(self, theta: float, phi: float = 0.0) -> CMatrix:
        """diag(S2, S1)(theta) by linear interpolation of the uniform table
        (DataTable::Sample, src/table.cpp:100-118)."""
        pos = (theta - 0.0) * self._inv_dx
        n = self._s1.size
        if pos <= 0.0:
            i, t = 0, 0.0
            s1, s2 = self._s1[0], self._s2[0]
        elif pos >= n - 1:
            s1, s2 = self._s1[-1], self._s2[-1]
        else:
            i = int(pos)
            t = pos - i
            s1 = self._s1[i] + t * (self._s1[i + 1] - self._s1[i])
            s2 = self._s2[i] + t * (self._s2[i + 1] - self._s2[i])
        out = CMatrix(2, 2)
        out[0, 0] = s2
        out[1, 1] = s1
        return out

    def scattering_cross_section(self) -> float:
        return self.phase_function.scattering_cross_section()

    def _amp_table(self, kind, n):
        s1 = np.zeros(2 * n)
        s2 = np.zeros(2 * n)
        N.check(N.lib().lmc_amplitude_table(kind, self.radius, self.n_particle, self.n_medium,
                                            self.wavelength, n, N.as_dptr(s1), N.as_dptr(s2)))
        self._set_amp(s1, s2, n)

    def _set_amp(self, s1, s2, n):
        self._s1 = s1.view(np.complex128)
        self._s2 = s2.view(np.complex128)
        self._dtheta = math.pi / (n - 1)
        self._inv_dx = 1.0 / self._dtheta


class RGDMedium(ScatteringMedium):
    """Rayleigh-Gans-Debye amplitudes on 2000 theta nodes (src/medium.cpp:77-120)."""

    def __init__(self, phase_func, radius, n_particle, n_medium, wavelength):
        super().__init__(phase_func)
        self.radius, self.n_particle = float(radius), float(n_particle)
        self.n_medium, self.wavelength = float(n_medium), float(wavelength)
        self.k = 2 * math.pi * self.n_medium / self.wavelength
        self._amp_table(N.AMP_RGD, 2000)


class MieMedium(ScatteringMedium):
    """Mie amplitudes on 1000 theta nodes at x = 2 pi r / lambda (src/medium.cpp:160-236)."""

    N_AMP = 1000

    def __init__(self, phase_func, radius, n_particle, n_medium, wavelength):
        self._set_particle(phase_func, radius, n_particle, n_medium, wavelength)
        self._amp_table(N.AMP_MIE, self.N_AMP)

    def _set_particle(self, phase_func, radius, n_particle, n_medium, wavelength):
        ScatteringMedium.__init__(self, phase_func)
        self.radius, self.n_particle = float(radius), float(n_particle)
        self.n_medium, self.wavelength = float(n_medium), float(wavelength)
        self.m = complex(self.n_particle / self.n_medium, 0.0)
        self.k = 2 * math.pi * self.n_medium / self.wavelength


def mie_species(species, nDiv=1000, minVal=0.0, maxVal=math.pi, timing=None):
    """Build many Mie species at once on the GPU (lmc_mie_tables).

    ``species`` is a sequence of (wavelength, radius, n_particle, n_medium).  Returns one
    (MiePhaseFunction(wavelength, radius, n_particle, n_medium, nDiv, minVal, maxVal),
    MieMedium(phase, radius, n_particle, n_medium, wavelength)) pair per species, with
    tables equal bit for bit to those the two constructors build one species at a time
    (src/phase.cpp:244-304, src/medium.cpp:160-236).  Needs a CUDA device.  ``timing``, a
    dict, receives the milliseconds of the host series, the uploads, the device kernels
    and the read-back.
    """
    species = [tuple(float(v) for v in q) for q in species]
    n = len(species)
    if int(nDiv) <= 0:
        raise ValueError("nDiv must be greater than 0")
    if not float(minVal) < float(maxVal):
        raise ValueError("minVal must be less than maxVal")
    arr = (N.MieSpecies * max(n, 1))(*[N.MieSpecies(*q) for q in species])
    n_amp = MieMedium.N_AMP
    values = np.zeros(int(nDiv) + 1)
    cdf = np.zeros((n, int(nDiv) + 1))
    sigma = np.zeros(max(n, 1))
    s1 = np.zeros((n, 2 * n_amp))
    s2 = np.zeros((n, 2 * n_amp))
    t_ms = np.zeros(4)
    N.check(N.lib().lmc_mie_tables(arr, n, int(nDiv), float(minVal), float(maxVal), n_amp,
                                   N.as_dptr(values), N.as_dptr(cdf), N.as_dptr(sigma),
                                   N.as_dptr(s1), N.as_dptr(s2), N.as_dptr(t_ms)))
    if timing is not None:
        timing.update(zip(("series_ms", "upload_ms", "kernels_ms", "readback_ms"), t_ms.tolist()))
    out = []
    for i, (wl, r, n_p, n_m) in enumerate(species):
        ph = MiePhaseFunction.__new__(MiePhaseFunction)
        ph._params = ph._set_particle(wl, r, n_p, n_m)
        ph._sigma = float(sigma[i])
        ph.nDiv, ph.minVal, ph.maxVal = int(nDiv), float(minVal), float(maxVal)
        ph._values, ph._cdf = values.copy(), cdf[i]
        med = MieMedium.__new__(MieMedium)
        med._set_particle(ph, r, n_p, n_m, wl)
        med._set_amp(s1[i], s2[i], n_amp)
        out.append((ph, med))
    return out


# ------------------------------------------------------------------------------ sample
class Layer:
    def __init__(self, z_min, z_max):
        self.z_min, self.z_max = float(z_min), float(z_max)

    def contains(self, z):
        return self.z_min <= z < self.z_max

    def thickness(self):
        return self.z_max - self.z_min


class SampleLayer(Layer):
    """HomogeneousLayer, bound as SampleLayer (python/python_module.cpp:557-559)."""

    def __init__(self, medium, z_min, z_max):
        super().__init__(z_min, z_max)
        self.medium = medium

    def mu_attenuation(self):
        return self.medium.mu_t

    def mu_scattering(self):
        return self.medium.mu_s

    def mu_absorption(self):
        return self.medium.mu_a


class MixtureLayer(Layer):
    """Several co-located species in one slab (include/luminis/core/sample.hpp:150-205,
    src/sample.cpp:41-104).  mu_s_i = n_i sigma_s_i from each species' phase-function
    scattering cross-section; the absorption keeps each species' albedo; free paths
    use mfp_total = 1 / mu_s_total; every vertex draws one uniform that selects a
    species on the normalised CDF of mu_s_i (last entry exactly 1)."""

    def __init__(self, species, number_densities, z_min, z_max):
        super().__init__(z_min, z_max)
        species = list(species)
        number_densities = [float(n) for n in number_densities]
        if not species:
            raise ValueError("MixtureLayer: species list must not be empty.")
        if len(species) != len(number_densities):
            raise ValueError("MixtureLayer: species and number_densities sizes differ.")
        self.species = species
        self.number_densities = number_densities
        self.mu_s_i = []
        mu_s_total = 0.0
        mu_a_total = 0.0
        for sp, n in zip(species, number_densities):
            if sp is None:
                raise ValueError("MixtureLayer: species pointer must not be null.")
            mu_s = n * sp.scattering_cross_section()
            self.mu_s_i.append(mu_s)
            mu_s_total += mu_s
            if sp.mu_s > 0.0:
                mu_a_total += mu_s * (sp.mu_a / sp.mu_s)
        if not mu_s_total > 0.0:
            raise ValueError("MixtureLayer: total mu_s must be positive (check number densities "
                             "and that the species' phase functions expose a scattering "
                             "cross-section).")
        self.mu_s_total = mu_s_total
        self.mu_a_total = mu_a_total
        self.mu_t_total = mu_s_total + mu_a_total
        self.mfp_total = 1.0 / mu_s_total
        self.selection_cdf = []
        acc = 0.0
        for mu_s in self.mu_s_i:
            acc += mu_s / mu_s_total
            self.selection_cdf.append(acc)
        self.selection_cdf[-1] = 1.0

    def mu_attenuation(self):
        return self.mu_t_total

    def mu_scattering(self):
        return self.mu_s_total

    def mu_absorption(self):
        return self.mu_a_total


class Sample:
    """Contiguous z-slabs from z = 0 sharing one host refractive index
    (include/luminis/core/sample.hpp:210-364, src/sample.cpp)."""

    def __init__(self, n_medium: float = 1.0):
        self.refractive_index = float(n_medium)
        self.light_speed = 1.0 / self.refractive_index
        self.layers: list[SampleLayer] = []
        self.interfaces: list[float] = []

    def _validate(self, z_min, z_max):                     # src/sample.cpp:120-140
        if z_max <= z_min:
            raise ValueError("Sample::add_layer: z_max must be greater than z_min.")
        if not self.layers:
            if z_min != 0.0:
                raise ValueError("Sample::add_layer: first layer must start at z = 0.")
            return
        prev = self.layers[-1].z_max
        if math.isinf(prev):
            raise ValueError("Sample::add_layer: cannot add a layer after an infinite top layer.")
        if z_min != prev:
            raise ValueError(f"Sample::add_layer: layer z_min ({z_min:f}) does not match previous "
                             f"z_max ({prev:f}).")

    def add_layer(self, medium, z_min, z_max):
        if medium is None:
            raise ValueError("Sample::add_layer: medium pointer must not be null.")
        z_min, z_max = float(z_min), float(z_max)
        self._validate(z_min, z_max)
        self.layers.append(SampleLayer(medium, z_min, z_max))
        if len(self.layers) > 1:
            self.interfaces.append(z_min)

    def add_mixture_layer(self, species, number_densities, z_min, z_max):
        z_min, z_max = float(z_min), float(z_max)
        self._validate(z_min, z_max)
        self.layers.append(MixtureLayer(species, number_densities, z_min, z_max))
        if len(self.layers) > 1:
            self.interfaces.append(z_min)

    def size(self):
        return len(self.layers)

    def get_layer(self, index):
        return self.layers[index]

    def light_speed_in_medium(self):
        return self.light_speed

    def z_top(self):
        return self.layers[-1].z_max if self.layers else 0.0

    def is_inside(self, position: Vec3) -> bool:
        if not self.layers:
            return False
        p = (position.x, position.y, position.z)
        if any(math.isnan(c) or math.isinf(c) for c in p):
            return False
        if position.z < 0.0:
            return False
        top = self.layers[-1].z_max
        return math.isinf(top) or position.z < top


# ------------------------------------------------------------------------------- laser
class Laser:
    """Photon source (include/luminis/core/laser.hpp:48-90, src/laser.cpp:29-40)."""

    def __init__(self, m_state, n_state, wavelength, sigma, source_type):
        self.position = Vec3(0.0, 0.0, 1e-9)
        self.polarization = CVec2(m_state, n_state)
        self.wavelength = float(wavelength)
        self.sigma = float(sigma)
        self.source_type = LaserSource(source_type)
        self.direction = Vec3(0, 0, 1)
        self.local_m = Vec3(1, 0, 0)
        self.local_n = Vec3(0, 1, 0)
        self.temporal_profile = TemporalProfile.Delta
        self.pulse_duration = 0.0
        self.repetition_rate = 0.0
        self.time_offset = 0.0

    def set_temporal_profile(self, profile, pulse_duration=0.0, repetition_rate=0.0,
                             time_offset=0.0):
        self.temporal_profile = TemporalProfile(profile)
        self.pulse_duration = float(pulse_duration)
        self.repetition_rate = float(repetition_rate)
        self.time_offset = float(time_offset)


def uniform_distribution(rng, center: Vec3, sigma: float) -> Vec3:
    theta = rng.uniform() * 2.0 * math.pi
    r = math.sqrt(rng.uniform()) * sigma
    return Vec3(center.x + r * math.cos(theta), center.y + r * math.sin(theta), center.z)


def gaussian_distribution(rng, center: Vec3, sigma: float) -> Vec3:
    return Vec3(rng.normal(center.x, sigma), rng.normal(center.y, sigma), center.z)


# ------------------------------------------------------------------------------ sensors
class Sensor:
    """Sensor base: plane z, absorption and filters (src/detector.cpp:314-417)."""
    _kind = -1
    _gpu = True

    def __init__(self, z: float, absorb: bool = True, estimator: bool = False):
        self.id = 0
        self.origin = Vec3(0, 0, z)
        self.normal = Vec3(0, 0, 1)
        self.backward_normal = Vec3(0, 0, -1)
        self.m_polarization = Vec3(1, 0, 0)
        self.n_polarization = Vec3(0, 1, 0)
        self.absorb_photons = bool(absorb)
        # estimator mode only exists at z == 0 (src/detector.cpp:323-331)
        self.estimator_enabled = bool(estimator) and z == 0.0
        self.hits = 0
        self.filter_theta_enabled = False
        self.filter_theta_min = self.filter_theta_max = 0.0
        self.filter_phi_enabled = False
        self.filter_phi_min = self.filter_phi_max = 0.0
        self.filter_position_enabled = False
        self.filter_x_min = self.filter_x_max = self.filter_y_min = self.filter_y_max = 0.0
        self.filter_direction_enabled = False
        self.filter_direction = CrossingDirection.Both
        self.filter_events_enabled = False
        self.filter_events_min = self.filter_events_max = 0
        self._tally = np.zeros(0)

    def set_theta_limit(self, min_theta, max_theta):
        self.filter_theta_enabled = True
        self.filter_theta_min, self.filter_theta_max = float(min_theta), float(max_theta)

    def set_phi_limit(self, min_phi, max_phi):
        self.filter_phi_enabled = True
        self.filter_phi_min, self.filter_phi_max = float(min_phi), float(max_phi)

    def set_position_limit(self, x_min, x_max, y_min, y_max):
        self.filter_position_enabled = True
        self.filter_x_min, self.filter_x_max = float(x_min), float(x_max)
        self.filter_y_min, self.filter_y_max = float(y_min), float(y_max)

    def set_direction_limit(self, direction):
        self.filter_direction_enabled = True
        self.filter_direction = CrossingDirection(direction)

    def set_events_limit(self, min_events, max_events):
        self.filter_events_enabled = True
        self.filter_events_min, self.filter_events_max = int(min_events), int(max_events)

    def _clone(self):
        """Deep copy with zeroed accumulators (Sensor::clone)."""
        c = copy.deepcopy(self)
        c._tally = np.zeros_like(self._tally)
        c.hits = 0
        return c

    def _shape(self):
        raise NotImplementedError

    def _grids(self, first_plane: int, n_planes: int):
        a = self._tally.reshape(self._shape())
        return [[a[p, t].view(Matrix) for t in range(a.shape[1])]
                for p in range(first_plane, first_plane + n_planes)]


class FarFieldCBSSensor(Sensor):
    """Coherent-backscattering far-field detector at z = 0, always absorbing
    (src/detector.cpp:851-907, process_hit :1231-1310)."""
    _kind = N.SENSOR_FARFIELD_CBS

    def __init__(self, theta_max, phi_max, len_t, d_theta, d_phi, d_t, estimator=False):
        super().__init__(0.0, True, estimator)
        self.theta_max, self.phi_max, self.t_max = float(theta_max), float(phi_max), float(len_t)
        self.dtheta, self.dphi, self.dt = float(d_theta), float(d_phi), float(d_t)
        self.N_t = 1 if self.dt == 0 else int(math.ceil(self.t_max / self.dt)) + 1
        self.N_theta = int(math.ceil(self.theta_max / self.dtheta))
        self.N_phi = int(math.ceil(self.phi_max / self.dphi))
        self.theta_pp_max = -1.0
        self.phi_explicit = False
        self.phi_values = [(j + 0.5) * self.dphi for j in range(self.N_phi)]
        self._tally = np.zeros(self._size())

    def _size(self):
        return 8 * self.N_t * self.N_theta * self.N_phi

    def _shape(self):
        return (8, self.N_t, self.N_theta, self.N_phi)

    def set_phi_slices(self, phi_angles):
        if not len(phi_angles):
            raise ValueError("set_phi_slices: phi_angles must be non-empty")
        for a in phi_angles:
            if a < 0.0 or a > 2.0 * math.pi:
                raise ValueError("set_phi_slices: every angle must be in [0, 2*pi]")
        self.phi_values = sorted(set(float(a) for a in phi_angles))
        self.phi_explicit = True
        self.N_phi = len(self.phi_values)
        self._tally = np.zeros(self._size())

    S0_coh = property(lambda self: self._grids(0, 1)[0])
    S1_coh = property(lambda self: self._grids(1, 1)[0])
    S2_coh = property(lambda self: self._grids(2, 1)[0])
    S3_coh = property(lambda self: self._grids(3, 1)[0])
    S0_incoh = property(lambda self: self._grids(4, 1)[0])
    S1_incoh = property(lambda self: self._grids(5, 1)[0])
    S2_incoh = property(lambda self: self._grids(6, 1)[0])
    S3_incoh = property(lambda self: self._grids(7, 1)[0])


class FarFieldFluenceSensor(Sensor):
    """Far-field forward-field Stokes |E_f|^2 on a (theta, phi) grid at z = 0.

    luminis-mc names this sensor in its documentation but ships no class for it;
    this one bins exits exactly as FarFieldCBSSensor (theta = acos(-s_z),
    phi = atan2(s_y, s_x) in [0, 2 pi), optional time axis with bin 0
    integrated) and accumulates the Stokes vector of the forward field alone,
    i.e. the CBS sensor's incoherent grid with no reverse path."""
    _kind = N.SENSOR_FARFIELD_FLUENCE

    def __init__(self, theta_max, phi_max, len_t, d_theta, d_phi, d_t):
        super().__init__(0.0, True, False)
        self.theta_max, self.phi_max, self.t_max = float(theta_max), float(phi_max), float(len_t)
        self.dtheta, self.dphi, self.dt = float(d_theta), float(d_phi), float(d_t)
        self.N_t = 1 if self.dt == 0 else int(math.ceil(self.t_max / self.dt)) + 1
        self.N_theta = int(math.ceil(self.theta_max / self.dtheta))
        self.N_phi = int(math.ceil(self.phi_max / self.dphi))
        self._tally = np.zeros(4 * self.N_t * self.N_theta * self.N_phi)

    def _shape(self):
        return (4, self.N_t, self.N_theta, self.N_phi)

    S0 = property(lambda self: self._grids(0, 1)[0])
    S1 = property(lambda self: self._grids(1, 1)[0])
    S2 = property(lambda self: self._grids(2, 1)[0])
    S3 = property(lambda self: self._grids(3, 1)[0])


class PlanarFluenceSensor(Sensor):
    """Time-resolved x-y Stokes grid (src/detector.cpp:704-841)."""
    _kind = N.SENSOR_PLANAR_FLUENCE

    def __init__(self, z, len_x, len_y, len_t, dx, dy, dt, absorb=True, estimator=False):
        super().__init__(float(z), absorb, estimator)
        self.len_x, self.len_y, self.len_t = float(len_x), float(len_y), float(len_t)
        self.dx, self.dy, self.dt = float(dx), float(dy), float(dt)
        self.N_t = 1 if self.dt == 0 else int(math.ceil(self.len_t / self.dt)) + 1
        self.N_x = int(math.ceil(self.len_x / self.dx))
        self.N_y = int(math.ceil(self.len_y / self.dy))
        self.set_position_limit(-0.5 * self.len_x, 0.5 * self.len_x, -0.5 * self.len_y,
                                0.5 * self.len_y)
        self._tally = np.zeros(4 * self.N_t * self.N_x * self.N_y)

    def _shape(self):
        return (4, self.N_t, self.N_x, self.N_y)

    S0 = property(lambda self: self._grids(0, 1)[0])
    S1 = property(lambda self: self._grids(1, 1)[0])
    S2 = property(lambda self: self._grids(2, 1)[0])
    S3 = property(lambda self: self._grids(3, 1)[0])


class PlanarFieldSensor(Sensor):
    """Complex field (speckle) grid (src/detector.cpp:490-568)."""
    _kind = N.SENSOR_PLANAR_FIELD

    def __init__(self, z, len_x, len_y, dx, dy, absorb=True, estimator=False):
        super().__init__(float(z), absorb, estimator)
        self.len_x, self.len_y = float(len_x), float(len_y)
        self.dx, self.dy = float(dx), float(dy)
        self.N_x = int(math.ceil(self.len_x / self.dx))
        self.N_y = int(math.ceil(self.len_y / self.dy))
        self.set_position_limit(-0.5 * self.len_x, 0.5 * self.len_x, -0.5 * self.len_y,
                                0.5 * self.len_y)
        self._tally = np.zeros(4 * self.N_x * self.N_y)

    def _shape(self):
        return (2, self.N_x, self.N_y, 2)

    @property
    def Ex(self):
        return self._tally.reshape(self._shape())[0].view(np.complex128)[..., 0].view(CMatrix)

    @property
    def Ey(self):
        return self._tally.reshape(self._shape())[1].view(np.complex128)[..., 0].view(CMatrix)


class PhotonRecordSensor(Sensor):
    """Per-photon snapshots at a plane.  Accepted for scene building; runs that
    include it raise NotImplementedError (the GPU path keeps no per-hit lists)."""
    _gpu = False

    def __init__(self, z, absorb=True):
        super().__init__(float(z), absorb, False)
        self.recorded_photons = []


class StatisticsSensor(Sensor):
    """Histograms of the photons crossing plane z (include/luminis/core/detector.hpp:595-699,
    src/detector.cpp:1569-1888): counts by scattering events, exit theta = acos(-s_z),
    exit phi, penetration depth, arrival time and weight.  Each histogram exists once its
    set_*_histogram_bins was called; events, theta, phi and depth have the time axis of
    set_time_resolution (slice 0 integrated, slices 1.. the windows of width dt)."""
    _kind = N.SENSOR_STATISTICS
    _NAMES = ("events", "theta", "phi", "depth", "time", "weight")

    def __init__(self, z, absorb=False):
        super().__init__(float(z), absorb, False)
        self.N_t, self.dt, self.t_max = 1, 0.0, 0.0
        for name in self._NAMES:
            setattr(self, f"{name}_histogram_bins_set", False)
        self.max_events = 0
        self.min_theta = self.max_theta = self.dtheta = 0.0
        self.n_bins_theta = 0
        self.min_phi = self.max_phi = self.dphi = 0.0
        self.n_bins_phi = 0
        self.max_depth = self.ddepth = 0.0
        self.n_bins_depth = 0
        self.h_max_time = self.h_dtime = 0.0
        self.n_bins_time = self._time_bins = 0
        self.max_weight = self.dweight = 0.0
        self.n_bins_weight = 0
        self._tally = np.zeros(0)

    # histogram sizes in layout order: (name, time slices, bins)
    def _parts(self):
        out = []
        for name, n in (("events", self.max_events), ("theta", self.n_bins_theta),
                        ("phi", self.n_bins_phi), ("depth", self.n_bins_depth)):
            if getattr(self, f"{name}_histogram_bins_set"):
                out.append((name, self.N_t, n))
        if self.time_histogram_bins_set:
            out.append(("time", 0, self._time_bins))
        if self.weight_histogram_bins_set:
            out.append(("weight", 0, self.n_bins_weight))
        return out

    def _reset(self):
        self._tally = np.zeros(sum(max(t, 1) * n for _, t, n in self._parts()))

    def _shape(self):
        return (self._tally.size,)

    def _hist(self, name):
        off = 0
        for nm, t, n in self._parts():
            size = max(t, 1) * n
            if nm == name:
                a = self._tally[off:off + size]
                return ([[int(v) for v in row] for row in a.reshape(t, n)] if t
                        else [int(v) for v in a])
            off += size
        return []

    events_histogram = property(lambda self: self._hist("events"))
    theta_histogram = property(lambda self: self._hist("theta"))
    phi_histogram = property(lambda self: self._hist("phi"))
    depth_histogram = property(lambda self: self._hist("depth"))
    time_histogram = property(lambda self: self._hist("time"))
    weight_histogram = property(lambda self: self._hist("weight"))

    def set_time_resolution(self, len_t, dt):                 # src/detector.cpp:1802-1834
        self.t_max, self.dt = float(len_t), float(dt)
        if self.dt <= 0.0:
            self.N_t, self.dt = 1, 0.0
        else:
            self.N_t = int(math.ceil(self.t_max / self.dt)) + 1
        self._reset()

    def set_events_histogram_bins(self, max_events):
        self.max_events = int(max_events)
        self.events_histogram_bins_set = True
        self._reset()

    def set_theta_histogram_bins(self, min_theta, max_theta, n_bins):
        self.min_theta, self.max_theta = float(min_theta), float(max_theta)
        self.n_bins_theta = int(n_bins)
        self.dtheta = (self.max_theta - self.min_theta) / self.n_bins_theta if n_bins else math.inf
        self.theta_histogram_bins_set = True
        self._reset()

    def set_phi_histogram_bins(self, min_phi, max_phi, n_bins):
        self.min_phi, self.max_phi, self.n_bins_phi = float(min_phi), float(max_phi), int(n_bins)
        self.dphi = (self.max_phi - self.min_phi) / self.n_bins_phi if n_bins else math.inf
        self.phi_histogram_bins_set = True
        self._reset()

    def set_depth_histogram_bins(self, max_depth, n_bins):
        self.max_depth, self.n_bins_depth = float(max_depth), int(n_bins)
        self.ddepth = self.max_depth / self.n_bins_depth if n_bins else math.inf
        self.depth_histogram_bins_set = True
        self._reset()

    def set_time_histogram_bins(self, max_time, n_bins):
        self.h_max_time = float(max_time)
        self._time_bins = int(n_bins)
        self.n_bins_time = max(1, int(n_bins))
        self.h_dtime = self.h_max_time / int(n_bins) if n_bins else math.inf
        self.time_histogram_bins_set = True
        self._reset()

    def set_weight_histogram_bins(self, max_weight, n_bins):
        self.max_weight, self.n_bins_weight = float(max_weight), int(n_bins)
        self.dweight = self.max_weight / self.n_bins_weight if n_bins else math.inf
        self.weight_histogram_bins_set = True
        self._reset()


class SensorsGroup:
    """Sensors indexed by plane (include/luminis/core/detector.hpp:726-761)."""

    def __init__(self):
        self.detectors: list[Sensor] = []

    def add_detector(self, detector: Sensor) -> Sensor:
        """Add a clone of `detector` and return the internal copy
        (python/python_module.cpp:318-322)."""
        c = detector._clone()
        c.id = len(self.detectors)
        self.detectors.append(c)
        return c


class Absorption:
    """Cylindrical absorption recorder (include/luminis/core/absortion.hpp:34-80,
    src/absortion.cpp).  Every scattering event deposits w mu_a / mu_t of its layer at
    the photon's position on an (r, z) grid of n_r = floor(radius/d_r)+1 by
    n_z = floor(depth/d_z)+1 cells; with d_t > 0 there are n_t = ceil(t_max/d_t)+1
    slices, slice 0 time-integrated and slice floor(t/d_t)+1 the arrival window.  The
    GPU transport deposits into a device grid that run_simulation_parallel adds to
    time_slices."""

    def __init__(self, radius, depth, d_r, d_z, d_t=0.0, t_max=0.0):
        self.radius, self.depth, self.d_r, self.d_z = map(float, (radius, depth, d_r, d_z))
        self.d_t, self.t_max = float(d_t), float(t_max)
        self.n_t = int(math.ceil(self.t_max / self.d_t)) + 1 if self.d_t > 0.0 else 1
        n_r = int(self.radius / self.d_r) + 1
        n_z = int(self.depth / self.d_z) + 1
        self.time_slices = [Matrix(n_r, n_z) for _ in range(self.n_t)]

    def clone(self) -> "Absorption":
        return Absorption(self.radius, self.depth, self.d_r, self.d_z, self.d_t, self.t_max)

    def merge_from(self, other: "Absorption") -> None:
        for k in range(self.n_t):
            self.time_slices[k] += other.time_slices[k]

    def _grid(self) -> np.ndarray:
        return np.stack([np.asarray(m) for m in self.time_slices])

    def _add(self, grid: np.ndarray) -> None:
        for k in range(self.n_t):
            self.time_slices[k] += grid[k]

    def record_absorption(self, photon, d_weight: float) -> None:
        """Host-side deposit of one event (src/absortion.cpp:54-91); `photon` needs pos,
        launch_time, opticalpath and velocity."""
        pos = photon.pos
        r = math.sqrt(pos.x * pos.x + pos.y * pos.y)
        z = pos.z
        if r > self.radius or z < 0.0 or z > self.depth:
            return
        i_r, i_z = int(math.floor(r / self.d_r)), int(math.floor(z / self.d_z))
        n_r, n_z = self.time_slices[0].shape
        if i_r >= n_r or i_z >= n_z:
            return
        self.time_slices[0][i_r, i_z] += d_weight
        if self.d_t > 0.0:
            t = photon.launch_time + photon.opticalpath / photon.velocity
            k = int(math.floor(t / self.d_t)) + 1
            if 1 <= k < self.n_t:
                self.time_slices[k][i_r, i_z] += d_weight

    def get_absorption_image(self, n_photons: int, time_index: int = 0) -> Matrix:
        """(2 n_r) x n_z image mirrored about the axis, per photon and voxel volume
        (src/absortion.cpp:93-119)."""
        if time_index < 0 or time_index >= self.n_t:
            return Matrix(0, 0)
        grid = np.asarray(self.time_slices[time_index])
        n_r, n_z = grid.shape
        image = Matrix(2 * n_r, n_z)
        for i in range(n_r):
            r_in, r_out = i * self.d_r, (i + 1) * self.d_r
            voxel = math.pi * (r_out * r_out - r_in * r_in) * self.d_z
            row = grid[i] / (float(n_photons) * voxel)
            image[n_r - i] = row
            if i != 0:
                image[n_r + i] = row
        return image

    def get_total_image(self, n_photons: int) -> Matrix:
        return self.get_absorption_image(n_photons, 0)
