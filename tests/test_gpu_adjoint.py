"""Likelihood-ratio derivatives on the GPU (lmc_run_adjoint, lmc_adjoint_contract).

* FP64: the outputs and every derivative row equal the oracle's FP64 estimator
  (oracle/lmc_oracle.c) on the same Philox stream, to 1e-9 of each row's largest
  entry.
* FP32: the same estimator in FP32 transport, within the FP32 tally tolerance of the
  parity tests (5 % of each row's largest entry per bin).
* The estimator agrees with central finite differences (relative step 1 %, common
  random numbers) of FP64 GPU runs, within the combined standard error over replicas.
* torch.autograd: backward through lr_transport returns J^T grad_out.
"""
import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import workloads as W
from luminis_mc_b200.adjoint import AdjointTransport, lr_transport
from oracle import pyoracle as O
from tests.test_oracle_adjoint import adjoint_scene

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-9
FP32_BIN_TOL = 5e-2
RADIAL = dict(radial_sensor=1, radial_bins=10, radial_max=5.0)


def _gpu(spec, n, seed, precision):
    cfg, _, keep = W.build(lm, spec)
    tr = AdjointTransport(cfg, **RADIAL)
    out, jac, st = tr.run(n, seed, precision=precision)
    tr.close()
    return out.cpu().numpy(), jac.cpu().numpy(), st


def _oracle(spec, n, seed, rng):
    _, o = O.Oracle(spec).run_adjoint(n, seed, rng=rng, **RADIAL)
    return o / n


def _rows_close(got, want, tol):
    for r in range(want.shape[0]):
        scale = max(float(np.abs(want[r]).max()), 1e-300)
        err = float(np.abs(got[r] - want[r]).max())
        assert err <= tol * scale, f"row {r}: max error {err:.3e} vs scale {scale:.3e}"


def test_fp64_adjoint_matches_oracle(cuda):
    spec = adjoint_scene()
    out, jac, st = _gpu(spec, 3000, 11, "fp64")
    ref = _oracle(spec, 3000, 11, "philox_u53")
    assert st["error_flags"] == 0
    _rows_close(np.vstack([out[None], jac]), ref, FP64_RTOL)


def test_fp32_adjoint_matches_oracle(cuda):
    spec = adjoint_scene()
    out, jac, st = _gpu(spec, 3000, 11, "fp32")
    ref = _oracle(spec, 3000, 11, "philox_u24")
    _rows_close(np.vstack([out[None], jac]), ref, FP32_BIN_TOL)


def test_adjoint_outputs_equal_the_plain_run_tallies(cuda):
    """The derivative variant transports the same photons as run_simulation_parallel:
    its total is the fluence grid's summed S0 and its CBS rows are the S0 grids."""
    spec = dict(adjoint_scene(), n_photons=4000, seed=21)
    cfg, hs, keep = W.build(lm, spec)
    lm.run_simulation_parallel(cfg, precision="fp64")
    out, _, _ = _gpu(spec, 4000, 21, "fp64")
    cbs = W.tally_arrays(hs[0], "farfield_cbs")
    flu = W.tally_arrays(hs[1], "planar_fluence")
    np.testing.assert_allclose(out[0] * 4000, flu[0, 0].sum(), rtol=1e-9)
    np.testing.assert_allclose(out[11:16] * 4000, cbs[0].ravel(), rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(out[16:21] * 4000, cbs[4].ravel(), rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("name", ["mu_a", "mu_s", "mfp", "g"])
def test_lr_matches_gpu_finite_differences(name, cuda):
    R, N, H = 8, 100_000, 0.01
    spec = adjoint_scene()
    cfg, _, keep = W.build(lm, spec)
    tr = AdjointTransport(cfg, **RADIAL)
    p0 = tr.parameters()
    idx = ("mu_a", "mu_s", "mfp", "g").index(name)
    zs = []
    for medium in range(2):
        v = p0[medium, idx]
        plus, minus = p0.copy(), p0.copy()
        plus[medium, idx] *= 1 + H
        minus[medium, idx] *= 1 - H
        lr, fd = [], []
        for r in range(R):
            seed = 500 + r
            tr.set_parameters(p0)
            lr.append(tr.run(N, seed, precision="fp64")[1][4 * medium + idx].cpu().numpy())
            tr.set_parameters(plus)
            hi = tr.run(N, seed, precision="fp64")[0].cpu().numpy()
            tr.set_parameters(minus)
            lo = tr.run(N, seed, precision="fp64")[0].cpu().numpy()
            fd.append((hi - lo) / (2 * H * v))
        lr, fd = np.array(lr), np.array(fd)
        for j in (0, 1, 2, 4, 11):
            a, b = lr[:, j], fd[:, j]
            se = np.sqrt(a.var(ddof=1) / R + b.var(ddof=1) / R)
            if se == 0:
                continue
            zs.append((a.mean() - b.mean()) / se)
    tr.close()
    zs = np.array(zs)
    assert np.all(np.abs(zs) < 4.5), zs
    assert np.mean(zs ** 2) < 3.0, zs


def test_autograd_backward_is_jacobian_transpose(cuda):
    import torch
    spec = adjoint_scene()
    cfg, _, keep = W.build(lm, spec)
    tr = AdjointTransport(cfg, **RADIAL)
    theta = torch.tensor(tr.parameters(), dtype=torch.float64, requires_grad=True)
    out = lr_transport(theta, tr, 5000, 3, precision="fp64")
    w = torch.linspace(-1.0, 1.0, out.numel(), dtype=torch.float64, device=out.device)
    (out * w).sum().backward()
    _, jac, _ = tr.run(5000, 3, precision="fp64")
    want = (jac.cpu() @ w.cpu()).view(theta.shape)
    np.testing.assert_allclose(theta.grad.numpy(), want.numpy(), rtol=1e-9,
                               atol=1e-12 * float(want.abs().max()))
    tr.close()


def test_set_parameters_round_trip(cuda):
    spec = adjoint_scene()
    cfg, _, keep = W.build(lm, spec)
    tr = AdjointTransport(cfg, **RADIAL)
    a, ja, _ = tr.run(2000, 5, precision="fp64")
    p = tr.parameters()
    tr.set_parameters(p * 1.1)
    tr.set_parameters(p)
    b, jb, _ = tr.run(2000, 5, precision="fp64")
    np.testing.assert_allclose(b.cpu().numpy(), a.cpu().numpy(), rtol=1e-12, atol=1e-15)
    tr.close()


def test_adjoint_rejects_inline_scenes(cuda):
    spec = adjoint_scene()
    spec["sensors"][1]["z"] = 0.25                 # a plane inside the sample
    cfg, _, keep = W.build(lm, spec)
    with pytest.raises(NotImplementedError):
        AdjointTransport(cfg, **RADIAL)
