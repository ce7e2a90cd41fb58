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


def test_batched_spectrum_matches_the_single_series_restatement():
    """The batched (torch, device-agnostic) spectrum and harmonic bands equal hhg_spectrum and
    harmonic_intensities run one series at a time (here on the CPU; "cuda" runs the same code)."""
    rng = np.random.default_rng(3)
    n_t, dt = 1500, 0.05
    t = np.arange(n_t) * dt
    w0s = [0.057, 0.045, 0.035]
    d = np.stack([np.sin(w0 * t) * np.sin(np.pi * t / t[-1]) ** 2 + 1e-3 * np.sin(7 * w0 * t)
                  + 1e-6 * rng.standard_normal(n_t) for w0 in w0s])
    w, spec = S.hhg_spectra_batched(d, dt, device="cpu")
    inten = S.harmonic_intensities_batched(w, spec, w0s, 15)
    for b, w0 in enumerate(w0s):
        w1, s1 = S.hhg_spectrum(d[b], dt)
        np.testing.assert_allclose(w, w1, rtol=0, atol=0)
        np.testing.assert_allclose(spec[b].numpy(), s1, rtol=1e-9, atol=1e-12 * s1.max())
        np.testing.assert_allclose(inten[b], S.harmonic_intensities(w1, s1, w0, 15), rtol=1e-9,
                                   atol=1e-12 * s1.max())


def test_spectrum_matches_the_reference_recipe():
    """Against the reference's own analysis.py lines (windowed, occupation-weighted total dipole with
    its l selection, 8th-order second derivative, padding, FFT), executed on seeded synthetic dipole
    files by tests/golden/make_spectrum_fixture.py."""
    import os
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "spectrum_analysis.npz"))
    d = z["dipole"]
    tot = S.total_dipole(d, z["l_active"], z["m_active"], z["occ"])
    win = tot * S.kaiser_periodic(tot.size, 24.0)
    assert np.abs(win - z["total_windowed"].real).max() <= 1e-13 * np.abs(z["total_windowed"]).max()
    w, spec = S.hhg_spectrum(tot, float(z["dt"]))
    ref = z["spectrum"]
    assert spec.shape == ref.shape
    assert np.abs(spec - ref).max() <= 1e-11 * ref.max()
