"""HHG spectrum of a dipole time series, as the reference's post-processing computes it.

Restates ``src/scripts/analysis.py``:

* window: Kaiser, beta = 24, periodic (``scipy.signal.windows.kaiser(N_t, beta=24, sym=False)``,
  analysis.py:200), applied to the occupation-weighted dipole before differentiation
  (analysis.py:433);
* total dipole of a single run: sum over orbitals of occ * Re d[l][kso], with l running from
  ``l_kso`` (if l_kso == 0 or l_kso == m_kso, else m_kso) to N_l - 5, l = l_kso excluded
  (analysis.py:400-435; Lext = N_l - 4, analysis.py:127);
* acceleration: 8th-order central finite-difference second derivative, zero on the four end
  points (``internal.d2fdx2``, internal.py:361-379);
* spectrum: zero padding of 8 N_t on each side, |fftshift(fft(fftshift(a)))|^2
  (analysis.py:147, 457-459).

Harmonic intensities are integrals of the spectrum over the band |w - q w0| < w0/2.
"""
from __future__ import annotations

from typing import Optional, Sequence, Tuple

import numpy as np


def kaiser_periodic(n: int, beta: float = 24.0) -> np.ndarray:
    """Periodic Kaiser window of length n (the symmetric window of length n + 1 without its last point)."""
    return np.kaiser(n + 1, beta)[:-1]


def d2fdx2(f: np.ndarray, dx: float) -> np.ndarray:
    """8th-order central second derivative; the 4 points at each end are 0 (internal.py:361-379)."""
    c4, c3, c2, c1, c0 = -1.0 / 560.0, 8.0 / 315.0, -0.20, 8.0 / 5.0, -205.0 / 72.0
    f = np.asarray(f, dtype=np.float64)
    out = np.zeros_like(f)
    k = slice(4, f.size - 4)
    out[k] = (c4 * (f[8:] + f[:-8]) + c3 * (f[7:-1] + f[1:-7]) + c2 * (f[6:-2] + f[2:-6])
              + c1 * (f[5:-3] + f[3:-5]) + c0 * f[4:-4])
    return out / dx ** 2


def total_dipole(dipole: np.ndarray, l_active: Sequence[int], m_active: Sequence[int],
                 occ: Sequence[float], reference_l_selection: bool = True) -> np.ndarray:
    """sum_kso occ_kso sum_l Re d[l][kso][t]  (dipole is [N_l][N_kso][N_t])."""
    n_l, n_kso, n_t = dipole.shape
    tot = np.zeros(n_t)
    for k in range(n_kso):
        if reference_l_selection:
            lk, mk = int(l_active[k]), int(m_active[k])
            lmin = lk if (lk == 0 or lk == mk) else mk
            ls = [l for l in range(lmin, n_l - 4) if l != lk]
        else:
            ls = list(range(n_l))
        tot += float(occ[k]) * dipole[ls, k, :].real.sum(axis=0)
    return tot


def hhg_spectrum(d_total: np.ndarray, dt: float, n_pad: int = 8, beta: float = 24.0,
                 window: bool = True) -> Tuple[np.ndarray, np.ndarray]:
    """(omega, |FFT of the windowed dipole's second derivative|^2), omega ascending."""
    n_t = d_total.size
    d = d_total * kaiser_periodic(n_t, beta) if window else d_total
    a = np.pad(d2fdx2(d, dt), n_pad * n_t, mode="constant")
    spec = np.abs(np.fft.fftshift(np.fft.fft(np.fft.fftshift(a)))) ** 2
    w = 2.0 * np.pi * np.fft.fftshift(np.fft.fftfreq(a.size, dt))
    return w, spec


def harmonic_intensities(w: np.ndarray, spec: np.ndarray, omega0: float, q_max: int) -> np.ndarray:
    """I_q = sum of the spectrum over |w - q w0| < w0/2, q = 1..q_max (positive frequencies)."""
    dw = w[1] - w[0]
    out = np.zeros(q_max)
    for q in range(1, q_max + 1):
        sel = np.abs(w - q * omega0) < 0.5 * omega0
        out[q - 1] = spec[sel].sum() * dw
    return out


def hhg_spectra_batched(d_totals, dt: float, n_pad: int = 8, beta: float = 24.0, window: bool = True,
                        device=None):
    """hhg_spectrum of several dipole series of one length at once, on ``device`` (torch: "cuda" runs
    the window, the derivative and one batched FFT on the GPU).  ``d_totals`` is [B][N_t] (NumPy or
    torch).  Returns (omega [n] NumPy, spec [B][n] torch on ``device``), n = (2 n_pad + 1) N_t."""
    import torch
    d = torch.as_tensor(np.asarray(d_totals, dtype=np.float64) if not torch.is_tensor(d_totals) else d_totals,
                        dtype=torch.float64, device=device)
    if d.dim() == 1:
        d = d[None]
    n_b, n_t = d.shape
    if window:
        d = d * torch.as_tensor(kaiser_periodic(n_t, beta), dtype=torch.float64, device=d.device)
    c4, c3, c2, c1, c0 = -1.0 / 560.0, 8.0 / 315.0, -0.20, 8.0 / 5.0, -205.0 / 72.0
    a = torch.zeros((n_b, (2 * n_pad + 1) * n_t), dtype=torch.float64, device=d.device)
    o = n_pad * n_t
    a[:, o + 4:o + n_t - 4] = (c4 * (d[:, 8:] + d[:, :-8]) + c3 * (d[:, 7:-1] + d[:, 1:-7])
                               + c2 * (d[:, 6:-2] + d[:, 2:-6]) + c1 * (d[:, 5:-3] + d[:, 3:-5])
                               + c0 * d[:, 4:-4]) / dt ** 2
    f = torch.fft.fftshift(torch.fft.fft(torch.fft.fftshift(a, dim=-1), dim=-1), dim=-1)
    spec = f.real ** 2 + f.imag ** 2
    w = 2.0 * np.pi * np.fft.fftshift(np.fft.fftfreq(a.shape[1], dt))
    return w, spec


def harmonic_intensities_batched(w: np.ndarray, spec, omega0s: Sequence[float], q_max: int) -> np.ndarray:
    """harmonic_intensities of each row of ``spec`` ([B][n] torch, any device) with its own omega0:
    the band |w - q w0| < w0/2 is a contiguous index range of the uniform grid w, summed on the
    device through a cumulative sum.  Returns [B][q_max] NumPy."""
    import torch
    dw = w[1] - w[0]
    n_b = spec.shape[0]
    lo = np.zeros((n_b, q_max), dtype=np.int64)
    hi = np.zeros((n_b, q_max), dtype=np.int64)
    for b in range(n_b):
        for q in range(1, q_max + 1):
            w0 = float(omega0s[b])
            lo[b, q - 1] = np.searchsorted(w, q * w0 - 0.5 * w0, side="right")   # first w > q w0 - w0/2
            hi[b, q - 1] = np.searchsorted(w, q * w0 + 0.5 * w0, side="left")    # first w >= q w0 + w0/2
    cs = torch.nn.functional.pad(torch.cumsum(spec, dim=-1), (1, 0))
    lo_t = torch.as_tensor(lo, device=spec.device)
    hi_t = torch.as_tensor(hi, device=spec.device)
    return ((cs.gather(1, hi_t) - cs.gather(1, lo_t)) * dw).cpu().numpy()


def cutoff_order(ip: float, e0: float, omega0: float) -> int:
    """Harmonic order of the semiclassical cutoff Ip + 3.17 Up, Up = E0^2 / (4 w0^2)."""
    up = e0 ** 2 / (4.0 * omega0 ** 2)
    return int(np.floor((ip + 3.17 * up) / omega0))


def harmonic_errors(spec_test: np.ndarray, spec_ref: np.ndarray, w: np.ndarray, omega0: float,
                    q_max: int) -> np.ndarray:
    """Relative error of each harmonic intensity, |I_q - I_q^ref| / I_q^ref, q = 1..q_max."""
    a = harmonic_intensities(w, spec_test, omega0, q_max)
    b = harmonic_intensities(w, spec_ref, omega0, q_max)
    return np.abs(a - b) / np.maximum(b, 1e-300)
