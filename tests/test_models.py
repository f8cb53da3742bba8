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
