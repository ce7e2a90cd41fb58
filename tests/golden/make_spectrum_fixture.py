"""Golden vectors of the reference's HHG-spectrum recipe (``src/scripts/analysis.py``).

The recipe is module-level script code in analysis.py, not a function, so this script executes the
reference's own lines: it reads the source text of analysis.py, takes the single-run block that
builds the windowed total dipole from the per-(orbital, l) dipole files (from
``dipoleMoment = np.zeros((N_kso, N_t), dtype=complex)`` through
``totalDipole = np.sum(dipoleMoment, axis=0)``, analysis.py:400-436) and the three spectrum lines
(``totalDipole = np.pad(internal.d2fdx2(...))`` .. ``spectrumTotal = ...``, analysis.py:457-459),
and runs them with the window of analysis.py:200 on seeded synthetic dipole files written in the
reference's output layout.  Plotting calls go to a stub.  The reference's ``internal`` module
(``d2fdx2``, ``getKSOL``/``getKSOM``) is imported from the reference tree with the NumPy shims it
needs (``np.complex``/``np.int`` were removed in NumPy 1.24).

Stored in ``tests/golden/spectrum_analysis.npz``: the per-l dipole d[l][kso][t], dt, targetID, occ,
the windowed total dipole and spectrumTotal.  ``tests/test_spectrum.py`` compares
``ggbtddft_b200.spectrum`` with them.

Usage:  python tests/golden/make_spectrum_fixture.py [<reference src directory>]
"""
import os
import shutil
import sys
import tempfile
import textwrap
from unittest import mock

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "spectrum_analysis.npz")

N_L, N_T, TARGET_ID, DT = 9, 320, 3, 0.05        # targetID 3: orbitals (l, m) = (0, 0), (1, 0), (1, 1)
OCC = np.array([2, 2, 4])


def _block(lines, start, stop, after=0):
    """Source lines from the first line (at or after index ``after``) that starts with ``start`` through
    the next one that starts with ``stop``, dedented; and the index of that last line."""
    i = next(k for k in range(after, len(lines)) if lines[k].strip().startswith(start))
    j = next(k for k in range(i, len(lines)) if lines[k].strip().startswith(stop))
    return textwrap.dedent("".join(lines[i:j + 1]).expandtabs(4)), j


def main(src):
    sys.path.insert(0, os.path.join(src, "scripts", "phys"))
    np.complex = complex
    np.int = int
    import internal                                   # noqa: E402  (the reference's module)
    from scipy.signal import windows
    lines = open(os.path.join(src, "scripts", "analysis.py")).readlines()
    build, end = _block(lines, "dipoleMoment = np.zeros((N_kso, N_t), dtype=complex)",
                        "totalDipole = np.sum(dipoleMoment")
    spec, _ = _block(lines, "totalDipole   = np.pad(internal.d2fdx2", "spectrumTotal = np.power", after=end)

    rng = np.random.default_rng(11)
    t = (np.arange(N_T) - N_T // 2) * DT
    env = np.exp(-np.power(t / (0.3 * N_T * DT), 2.0))
    n_kso = 3
    d = np.zeros((N_L, n_kso, N_T), dtype=np.complex128)
    for l in range(N_L):
        for k in range(n_kso):
            w = rng.uniform(0.02, 3.0, 6)
            a = rng.standard_normal(6) * np.exp(-0.3 * l)
            d[l, k] = env * (a[:, None] * np.cos(w[:, None] * t[None, :] + rng.uniform(0, 6.3, 6)[:, None])).sum(0) \
                + 1j * rng.standard_normal(N_T) * 1e-3
    work = tempfile.mkdtemp(prefix="ggb_spec_")
    try:
        base = os.path.join(work, "timeDependent", "observables", "dipoleMoment", "scan000")
        for k in range(n_kso):
            os.makedirs(os.path.join(base, f"kso{k:03d}"))
            for l in range(N_L):
                d[l, k].astype(np.complex128).tofile(os.path.join(base, f"kso{k:03d}", f"dipL{l:03d}.bin"))
        ns = dict(np=np, internal=internal, plib=mock.MagicMock(), N_kso=n_kso, N_t=N_T, Lext=N_L - 4,
                  targetID=TARGET_ID, occ=OCC, filterDIP=windows.kaiser(N_T, beta=24, sym=False),
                  outputPath=work, dipMomentFigurePath=work, t=t, scalingT=1.0, N_pad=8, dt=DT, print=lambda *a: None)
        exec(build, ns)
        total = ns["totalDipole"].copy()
        exec(spec, ns)
    finally:
        shutil.rmtree(work, ignore_errors=True)
    np.savez_compressed(OUT, dipole=d, dt=DT, target_id=TARGET_ID, occ=OCC,
                        l_active=internal.getKSOL(TARGET_ID), m_active=internal.getKSOM(TARGET_ID),
                        total_windowed=total, spectrum=ns["spectrumTotal"])
    print("wrote", OUT)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/src")
