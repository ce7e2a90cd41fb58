"""The batched HHG spectrum on the GPU equals the single-series CPU restatement."""
import numpy as np
import pytest

from ggbtddft_b200 import spectrum as S

pytestmark = pytest.mark.gpu


def test_batched_spectrum_on_the_gpu():
    rng = np.random.default_rng(5)
    n_t, dt = 4000, 0.03
    t = np.arange(n_t) * dt
    w0s = [0.057, 0.04]
    d = np.stack([np.sin(w0 * t) * np.sin(np.pi * t / t[-1]) ** 2 + 1e-3 * np.sin(9 * w0 * t)
                  + 1e-6 * rng.standard_normal(n_t) for w0 in w0s])
    w, spec = S.hhg_spectra_batched(d, dt, device="cuda")
    assert spec.is_cuda
    inten = S.harmonic_intensities_batched(w, spec, w0s, 21)
    spec = spec.cpu().numpy()
    for b, w0 in enumerate(w0s):
        w1, s1 = S.hhg_spectrum(d[b], dt)
        np.testing.assert_allclose(spec[b], s1, rtol=1e-8, atol=1e-10 * s1.max())
        np.testing.assert_allclose(inten[b], S.harmonic_intensities(w1, s1, w0, 21), rtol=1e-8,
                                   atol=1e-10 * s1.max())
