"""HHG spectrum recipe (CPU): window, finite differences, harmonic bands."""
import numpy as np
import scipy.signal

from ggbtddft_b200 import spectrum as S


def test_kaiser_matches_scipy_periodic_window():
    for n in (16, 255, 1024):
        assert np.allclose(S.kaiser_periodic(n, 24.0), scipy.signal.windows.kaiser(n, beta=24, sym=False), atol=1e-14)


def test_second_derivative_exact_for_polynomials():
    t = np.linspace(0.0, 1.0, 101)
    dt = t[1] - t[0]
    f = 3.0 * t ** 2 - t ** 5
    d = S.d2fdx2(f, dt)
    assert np.allclose(d[4:-4], (6.0 - 20.0 * t ** 3)[4:-4], atol=1e-7)
    assert np.all(d[:4] == 0) and np.all(d[-4:] == 0)


def test_harmonic_band_of_a_pure_tone():
    dt, n, w0 = 0.05, 2 ** 15, 0.057       # ~15 optical cycles: the Kaiser(24) main lobe fits one band
    t = np.arange(n) * dt
    d = np.cos(3 * w0 * t)
    w, spec = S.hhg_spectrum(d, dt)
    iq = S.harmonic_intensities(w, spec, w0, 5)
    assert np.argmax(iq) == 2
    assert iq[2] > 1e4 * max(iq[0], iq[4])


def test_reference_l_selection():
    d = np.ones((10, 2, 3), dtype=complex)
    tot = S.total_dipole(d, l_active=[0, 1], m_active=[0, 1], occ=[2, 4])
    # kso 0: l = 1..5 (l = 0 excluded) -> 5 terms x 2; kso 1: l_kso == m_kso -> from 1, l = 2..5 -> 4 terms x 4
    assert np.allclose(tot, 5 * 2 + 4 * 4)
