"""Model and state utilities of the public API (``src/models/tfim.jl:50-76``,
``src/states/finite.jl:53-72``), on the CPU: the exact diagonalisation against
the oracle's restatement, and ``validate_state``'s checks on host stand-ins of
device states."""
import numpy as np
import pytest

from oracle import model as md


@pytest.mark.parametrize("Lx,Ly,h", [(2, 2, 0.7), (3, 2, 3.0), (3, 3, 1.3)])
def test_exact_diagonalization_matches_oracle(sps, Lx, Ly, h):
    H = sps.dense_hamiltonian(sps.Lattice(Lx, Ly), sps.TFIM(1.0, h))
    np.testing.assert_array_equal(H, md.dense_hamiltonian(Lx, Ly, md.TFIM(1.0, h)))
    for beta in (0.0, 0.3, 1.0):
        a = sps.exact_thermal_observables(sps.Lattice(Lx, Ly), sps.TFIM(1.0, h), beta)
        b = md.exact_thermal_observables(Lx, Ly, md.TFIM(1.0, h), beta)
        for k in ("energy_total", "energy_per_site", "lnZ"):
            assert abs(a[k] - b[k]) <= 1e-12 * max(1.0, abs(b[k]))
    assert abs(sps.exact_thermal_observables(sps.Lattice(Lx, Ly), sps.TFIM(1.0, h), 0.0)["lnZ"]
               - Lx * Ly * np.log(2)) < 1e-12
    assert sps.physical_space(sps.TFIM(1.0, h)) == sps.Z2Space(1, 1)


def test_per_site_fields_config_and_exact_diagonalization(sps):
    """The per-site-field extension: ED equals the oracle's, the uniform field
    written out per site gives the reference's model bit for bit, the config
    encoding of the reference's model is unchanged, and bad fields are refused."""
    rng = np.random.default_rng(3)
    f = tuple(0.7 + rng.uniform(-0.3, 0.3, 6))
    H = sps.dense_hamiltonian(sps.Lattice(3, 2), sps.TFIM(1.0, 0.7, fields=f))
    np.testing.assert_array_equal(H, md.dense_hamiltonian(3, 2, md.TFIM(1.0, 0.7, f)))
    np.testing.assert_array_equal(sps.dense_hamiltonian(sps.Lattice(3, 2), sps.TFIM(1.0, 0.7, fields=[0.7] * 6)),
                                  sps.dense_hamiltonian(sps.Lattice(3, 2), sps.TFIM(1.0, 0.7)))
    # d lnZ / d h_i = beta <X_i>: the field gradient is the site magnetization
    beta, i, eps = 0.4, 4, 1e-5
    def lnz(fi):
        g = list(f)
        g[i] = fi
        return sps.exact_thermal_observables(sps.Lattice(3, 2), sps.TFIM(1.0, 0.7, fields=g), beta)["lnZ"]
    w, v = np.linalg.eigh(H)
    rho = (v * np.exp(-beta * (w - w.min()))) @ v.T
    b = np.arange(64)
    xi = np.zeros((64, 64))
    xi[b ^ (1 << i), b] = 1.0
    assert abs((lnz(f[i] + eps) - lnz(f[i] - eps)) / (2 * eps) - beta * np.trace(rho @ xi) / np.trace(rho)) < 1e-7
    assert "fields" not in sps.parameter_dict(sps.RunConfig(lattice=sps.Lattice(3, 2)))["model"]
    assert sps.parameter_dict(sps.RunConfig(lattice=sps.Lattice(3, 2),
                                            model=sps.TFIM(fields=f)))["model"]["fields"] == list(f)
    with pytest.raises(ValueError):
        sps.TFIM(fields=[1.0, float("nan")])
    with pytest.raises(ValueError):
        sps.validate_config(sps.RunConfig(lattice=sps.Lattice(3, 2), model=sps.TFIM(fields=[1.0] * 5)))


class _HostState:
    """A host stand-in with the device state's interface (lattice, is_pepo, download)."""

    def __init__(self, Lx, Ly, D=2, pepo=False):
        self.lattice = (Lx, Ly)
        self.is_pepo = pepo
        self.dims = np.zeros((Lx * Ly, 6, 2), np.int32)
        for y in range(Ly):
            for x in range(Lx):
                d = self.dims[x + y * Lx]
                d[0] = (1, 0) if x == 0 else (D // 2, D // 2)
                d[1] = (1, 0) if y == 0 else (D // 2, D // 2)
                d[2] = (1, 1)
                d[3] = (1, 1) if pepo else (1, 0)
                d[4] = (1, 0) if x == Lx - 1 else (D // 2, D // 2)
                d[5] = (1, 0) if y == Ly - 1 else (D // 2, D // 2)
        self.sites = [np.ones([int(a + b) for a, b in d]) for d in self.dims]

    def download(self):
        return self.sites, self.dims


def test_validate_state_checks(sps):
    ok = _HostState(3, 2)
    assert sps.validate_state(ok) is ok
    sps.validate_state(_HostState(2, 3, pepo=True))
    bad = _HostState(3, 2)
    bad.sites[1][0, 0, 0, 0, 0, 0] = np.nan
    with pytest.raises(ValueError, match="nonfinite tensor at"):
        sps.validate_state(bad)
    bad = _HostState(3, 2)
    bad.dims[0][0] = (1, 1)
    with pytest.raises(ValueError, match="nontrivial OBC leg"):
        sps.validate_state(bad)
    bad = _HostState(3, 2)
    bad.dims[0][4] = (2, 1)
    with pytest.raises(ValueError, match="horizontal space mismatch"):
        sps.validate_state(bad)
    bad = _HostState(3, 2)
    bad.dims[1][5] = (2, 1)
    with pytest.raises(ValueError, match="vertical space mismatch"):
        sps.validate_state(bad)
    bad = _HostState(3, 2)
    bad.dims[2][3] = (1, 1)
    with pytest.raises(ValueError, match="PEPS auxiliary leg"):
        sps.validate_state(bad)
