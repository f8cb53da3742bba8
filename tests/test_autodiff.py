"""The torch.autograd wiring of ``LognormFunction`` (the Python counterpart
of a ChainRulesCore rrule around the device's lognorm derivative), on the
CPU: the engine is a stand-in whose lognorm derivative is the oracle's, so
the test checks the host plumbing only (argument slots, cotangent scaling,
the upload layout) against central finite differences of lognorm."""
import copy

import numpy as np
import torch

from oracle import adjoint as ad, boundary as bm, driver as dr
from oracle.z2 import T


class _State:
    def __init__(self, sites, dims, beta, log_amplitude):
        self.sites, self.dims, self.beta, self.log_amplitude = sites, dims, beta, log_amplitude


class _Engine:
    """Holds the uploaded arrays; the oracle state they stand for is rebuilt
    from a template with the same legs."""

    def __init__(self, template):
        self.template = template
        self.Lx, self.Ly = template.Lx, template.Ly

    def upload_state(self, sites, leg_dims, is_pepo, beta=0.0, log_amplitude=0.0):
        assert is_pepo
        st = copy.copy(self.template)
        st.sites = [[T(np.asarray(sites[x + y * self.Lx]), self.template[x, y].p) for y in range(self.Ly)]
                    for x in range(self.Lx)]
        st.log_amplitude = log_amplitude
        return st


def _fake_gradient(state, contraction, checkpoint_rows=False):
    value, g = ad.lognorm_with_gradient(state, contraction.chi)
    return value, [g[i % state.Lx][i // state.Lx] for i in range(state.Lx * state.Ly)]


def test_autograd_function_matches_finite_differences(sps, monkeypatch):
    from importlib import import_module
    autodiff = import_module(sps.__name__ + ".autodiff")
    monkeypatch.setattr(autodiff, "lognorm_gradient", _fake_gradient)
    c = dr.RunConfig(Lx=3, Ly=2, J=1.0, h=1.0, beta0=0.3, beta_log=[0.3], beta_measure=[0.3],
                     delta_tau_pur=0.05, D_pur=2, D_peps=2, chi_environment=64, Ns=1)
    st = dr.run_purification(c)[0]
    eng = _Engine(st)
    sites = [torch.tensor(st[i % 3, i // 3].a, dtype=torch.float64, requires_grad=True) for i in range(6)]
    m = sps.BoundaryMPS(6)
    out = autodiff.lognorm_differentiable(eng, sites, None, m, log_amplitude=st.log_amplitude)
    assert abs(out.item() - bm.lognorm(st, bm.BoundaryMPS(6))["log_norm"]) < 1e-12
    grads = torch.autograd.grad(3.0 * out, sites)
    rng = np.random.default_rng(5)
    dirs = [rng.standard_normal(s.shape) * (st[i % 3, i // 3].a != 0) for i, s in enumerate(sites)]
    eps = 1e-5

    def lz(sign):
        s2 = copy.copy(st)
        s2.sites = [[T(st[x, y].a + sign * eps * dirs[x + 3 * y], st[x, y].p) for y in range(2)] for x in range(3)]
        return bm.lognorm(s2, bm.BoundaryMPS(6))["log_norm"]

    fd = 3.0 * (lz(1) - lz(-1)) / (2 * eps)
    adj = sum(float((g.numpy() * d).sum()) for g, d in zip(grads, dirs))
    assert abs(fd - adj) <= 1e-7 * abs(fd)
