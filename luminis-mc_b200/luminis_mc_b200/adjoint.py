"""Differentiable transport: likelihood-ratio derivatives behind torch.autograd.

The transport kernel carries, per photon, the score s = d log(path density x
weight) / d theta of its history. That score sums the free-flight densities
(exponential with the medium's mean free path, rescaled by the mu_t ratio at
interfaces), the albedo factors mu_s / mu_t and the Henyey-Greenstein angle
densities. Every detected contribution v adds v * s_k to the derivative of its
output. This is a forward-mode estimate of the full Jacobian of the outputs with
respect to theta, made in the same pass as the outputs and from running per-photon
sums. The backward pass is then one contraction, grad_theta = J^T grad_out, done
by a CUDA kernel (lmc_adjoint_contract).

Parameters theta, per medium m in scene order: (mu_a, mu_s, mean_free_path, g);
g applies to media whose phase function is Henyey-Greenstein (its derivative is
zero otherwise). Outputs, per photon:
  * with a radial sensor (a PlanarFluenceSensor): the total S0 of its
    time-integrated grid, then `radial_bins` bins of the same S0 by hit radius;
  * for every FarFieldCBSSensor: S0 coherent and S0 incoherent, [N_t][N_theta][N_phi].

The reference has no derivatives; the estimator is checked against central
finite differences with common random numbers and against the FP64 oracle.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .simulation import SimConfig, scene_desc

PARAM_NAMES = ("mu_a", "mu_s", "mean_free_path", "g")


class AdjointTransport:
    """A scene whose medium parameters can be set per run, with derivative outputs."""

    def __init__(self, config: SimConfig, radial_sensor=None, radial_bins: int = 100,
                 radial_max: float = 5.0, device="cuda:0"):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        self.config = config
        self.scene, self._keep, self.sensors = scene_desc(config)
        if radial_sensor is not None and not isinstance(radial_sensor, int):
            radial_sensor = next(i for i, s in enumerate(self.sensors) if s is radial_sensor)
        self.opts = N.AdjointOpts(-1 if radial_sensor is None else int(radial_sensor),
                                  int(radial_bins), float(radial_max))
        self.n_media = self.scene.n_media
        self.n_params = 4 * self.n_media
        self._hg = [self.scene.media[m].theta_kind == N.THETA_HG for m in range(self.n_media)]
        self._handle = None
        self.n_out = None
        self._create()

    def _create(self):
        if self._handle is not None:
            N.lib().lmc_destroy(self._handle)
            self._handle = None
        with self.torch.cuda.device(self.device):
            h = C.c_void_p()
            N.check(N.lib().lmc_create(C.byref(self.scene), C.byref(h)))
        self._handle = h
        total, n_out, k = C.c_size_t(), C.c_size_t(), C.c_int()
        N.check(N.lib().lmc_tally_layout(h, -1, None, C.byref(total), None))
        N.check(N.lib().lmc_adjoint_layout(h, C.byref(self.opts), C.byref(n_out), C.byref(k)))
        self.tally_size = int(total.value)
        self.n_out = int(n_out.value)

    def parameters(self) -> np.ndarray:
        """Current theta as an [n_media, 4] array (mu_a, mu_s, mean_free_path, g)."""
        p = np.zeros((self.n_media, 4))
        for m in range(self.n_media):
            d = self.scene.media[m]
            p[m] = (d.mu_a, d.mu_s, d.mean_free_path, d.hg_g)
        return p

    def set_parameters(self, theta) -> None:
        theta = np.asarray(theta, dtype=np.float64).reshape(self.n_media, 4)
        for m in range(self.n_media):
            d = self.scene.media[m]
            d.mu_a, d.mu_s, d.mean_free_path = (float(x) for x in theta[m, :3])
            if self._hg[m]:
                d.hg_g = float(theta[m, 3])
        self._create()

    def layout(self) -> dict:
        """Slices of the output vector by name."""
        out, o = {}, 0
        if self.opts.radial_sensor >= 0:
            out["total"] = slice(0, 1)
            out["radial"] = slice(1, 1 + self.opts.radial_bins)
            o = 1 + self.opts.radial_bins
        for i, s in enumerate(self.sensors):
            if type(s).__name__ != "FarFieldCBSSensor":
                continue
            n = s.N_t * s.N_theta * s.N_phi
            out[f"cbs{i}_coherent"] = slice(o, o + n)
            out[f"cbs{i}_incoherent"] = slice(o + n, o + 2 * n)
            o += 2 * n
        return out

    def run(self, n_photons: int, seed: int, precision: str = "fp32", begin: int = 0,
            stream=None, tally_mode="default"):
        """(outputs [n_out], jacobian [n_params, n_out], stats), per photon, on the device.
        The run's sensor tallies stay in self.last_tallies (device, flat)."""
        torch = self.torch
        with torch.cuda.device(self.device):
            adj = torch.zeros((1 + self.n_params) * self.n_out, dtype=torch.float64,
                              device=self.device)
            tallies = torch.zeros(max(self.tally_size, 1), dtype=torch.float64, device=self.device)
            o = N.RunOpts()
            o.precision = N.PRECISION[precision]
            o.max_events = int(self.config.MAX_EVENTS)
            o.track_reverse_paths = int(bool(self.config.track_reverse_paths))
            o.stream = N.launch_stream(stream)
            o.tally_mode = N.tally_mode_value(tally_mode)
            st = N.Stats()
            torch.cuda.synchronize(self.device)
            N.check(N.lib().lmc_run_adjoint(self._handle, int(seed) & (2 ** 64 - 1), int(begin),
                                            int(n_photons), C.byref(o), C.byref(self.opts),
                                            C.c_void_p(tallies.data_ptr()),
                                            C.c_void_p(adj.data_ptr()), C.byref(st)))
        self.last_tallies = tallies
        adj = adj.view(1 + self.n_params, self.n_out) / float(max(n_photons, 1))
        return adj[0], adj[1:], st.as_dict()

    def close(self):
        if self._handle is not None:
            N.lib().lmc_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def contract(jacobian, grad_out):
    """grad_theta = J^T grad_out on the device (lmc_adjoint_contract)."""
    import torch
    J = jacobian.contiguous()
    g = grad_out.to(dtype=torch.float64).contiguous()
    K, n_out = J.shape
    # the kernel reads rows 1..K of a (1 + K) x n_out block: prepend an unused row
    block = torch.cat([torch.zeros(1, n_out, dtype=torch.float64, device=J.device), J])
    grad = torch.empty(K, dtype=torch.float64, device=J.device)
    N.check(N.lib().lmc_adjoint_contract(C.c_void_p(block.data_ptr()), C.c_void_p(g.data_ptr()),
                                         n_out, K, C.c_void_p(grad.data_ptr()),
                                         C.c_void_p(torch.cuda.current_stream(J.device).cuda_stream)))
    return grad


def _function():
    import torch

    class LRTransport(torch.autograd.Function):
        """outputs = T(theta); backward: J^T grad_out with J from the same pass."""

        @staticmethod
        def forward(ctx, theta, transport, n_photons, seed, precision):
            transport.set_parameters(theta.detach().cpu().numpy())
            out, jac, _ = transport.run(n_photons, seed, precision=precision)
            ctx.save_for_backward(jac)
            ctx.shape = theta.shape
            ctx.dtype = theta.dtype
            ctx.device = theta.device
            return out.to(theta.device)

        @staticmethod
        def backward(ctx, grad_out):
            (jac,) = ctx.saved_tensors
            g = contract(jac, grad_out.to(jac.device))
            return g.view(ctx.shape).to(device=ctx.device, dtype=ctx.dtype), None, None, None, None

    return LRTransport


_LR = None


def lr_transport(theta, transport: AdjointTransport, n_photons: int, seed: int,
                 precision: str = "fp32"):
    """Differentiable outputs of `transport` at parameters theta ([n_media, 4] tensor,
    requires_grad as needed): returns the per-photon output vector (see layout())."""
    global _LR
    if _LR is None:
        _LR = _function()
    return _LR.apply(theta, transport, n_photons, seed, precision)
