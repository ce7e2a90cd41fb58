"""The ground-state SCF's device-resident loop (torch, run here on the CPU device) against the
NumPy host loop: same iteration, same fixed point."""
import numpy as np
import pytest

from ggbtddft_b200 import inputs as I


@pytest.mark.parametrize("atom,Z,orbitals,n_r,r_max", [
    ("He", 2.0, I.ORBITALS_HE, 150, 80.0),
    ("Ar", 18.0, I.ORBITALS_AR, 200, 100.0),
])
def test_device_loop_matches_host_loop(atom, Z, orbitals, n_r, r_max):
    g = I.make_grid(n_r, r_max, I.zeta_physical_to_ref(0.5, r_max))
    a = I.ground_state(g, Z, orbitals, True, correlation=True)
    b = I.ground_state(g, Z, orbitals, True, correlation=True, device="cpu")
    assert np.abs(a.vscf - b.vscf).max() < 1e-10
    assert np.abs(a.energies - b.energies).max() < 1e-10 * np.abs(a.energies).max()
    assert np.abs(a.u - b.u).max() < 1e-10
    # occupied levels in order, and the potential self-consistent
    assert np.all(np.diff(sorted(b.energies)) >= -1e-12)


def test_device_loop_one_electron():
    g = I.make_grid(120, 60.0, I.zeta_physical_to_ref(0.5, 60.0))
    a = I.ground_state(g, 1.0, I.ORBITALS_H, False)
    b = I.ground_state(g, 1.0, I.ORBITALS_H, False, device="cpu")
    assert abs(a.energies[0] - b.energies[0]) < 1e-12
    assert abs(a.energies[0] + 0.5) < 1e-6
    assert np.abs(a.u - b.u).max() < 1e-12
    assert np.all(b.vscf == 0.0)
