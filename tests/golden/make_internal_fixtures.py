"""Golden vectors of the reference's own input producers (``src/scripts/phys/internal.py``).

Runs the reference's functions themselves -- imported from the reference tree, not restated -- on
small inputs and stores what they return or write:

    generateGaussLobattoGrid (internal.py:524-556)   r, drdx, T, P of N_r = 32 (shipped roots file)
    getABCR, ABC_TYPE = 1      (internal.py:447-497)  the Manolopoulos CAP on that grid
    propagatorsR, CN           (internal.py:232-333)  propagatorL%03d.bin for l < N_l, from the
                                                      potentials v0 (with -i CAP, as groundState.py:27
                                                      builds it) and vscf stored beside them
    propagatorsL, LDX = 1, 2, 3 (internal.py:122-198) V%03d.bin / D%03d.bin of P, FP, D and FF per m

into ``tests/golden/internal_inputs.npz``.  ``tests/test_inputs_vs_reference.py`` compares
``ggbtddft_b200.inputs`` with them.  Needs the reference sources (this container only) and the one
shim ``internal.py`` needs under NumPy >= 1.24 (``np.complex`` was removed; it is ``complex``).  The
functions write their files relative to the working directory, so they run in a temporary copy of
the directory tree they expect; the reference tree is only read.

Usage:  python tests/golden/make_internal_fixtures.py [<reference src directory>]
"""
import contextlib
import io
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "internal_inputs.npz")

N_R, N_L, N_M = 32, 6, 3          # radial grid, propagators' N_l, m = 0..N_M-1 of the angular systems
N_L_ANG = 12                      # N_l of the angular eigensystems
R_MAX, R_MASK, ZETA = 45.0, 30.0, 0.5
DT = 0.05


def main(src):
    sys.path.insert(0, os.path.join(src, "scripts", "phys"))
    np.complex = complex                      # removed from NumPy 1.24; internal.py:260,450,536 use it
    import internal                           # noqa: E402  (the reference's module)
    work = tempfile.mkdtemp(prefix="ggb_internal_")
    cwd = os.getcwd()
    try:
        os.makedirs(os.path.join(work, "workingData", "mesh", "legendreRoots"))
        shutil.copy(os.path.join(src, "workingData", "mesh", "legendreRoots", f"roots{N_R:05d}.txt"),
                    os.path.join(work, "workingData", "mesh", "legendreRoots"))
        os.makedirs(os.path.join(work, "workingData", "hamiltonian", "propagators"))
        for d in ("001/001", "001/003", "002/002", "003/003"):
            os.makedirs(os.path.join(work, "workingData", "hamiltonian", "propagatorsL", d))
        os.chdir(work)
        r, drdx, d, T, N_g, x, P, D1 = internal.generateGaussLobattoGrid(N_R, R_MASK, R_MAX, ZETA)
        cap = internal.getABCR(r, R_MASK, R_MAX, 1)
        # potentials as the reference's ground state hands them to propagatorsR: v0 = -Z/r - i W
        # (groundState.py:27) and a smooth real self-consistent part
        v0 = -1.0 / r - 1j * cap.real
        vscf = 0.8 * np.exp(-0.5 * r) / (1.0 + r)
        with contextlib.redirect_stdout(io.StringIO()):
            internal.propagatorsR(r, T, v0, vscf, cap.real, np.array([0]), N_R, N_L, DT, 0, R_MASK)
        W = np.stack([np.fromfile(f"workingData/hamiltonian/propagators/propagatorL{l:03d}.bin",
                                  dtype=np.complex128).reshape(N_R, N_R) for l in range(N_L)])
        for ldx in (1, 2, 3):
            internal.propagatorsL(np.arange(N_M), N_L_ANG, ldx)
        ang = {}
        for name, path in (("P", "001/001"), ("FP", "001/003"), ("D", "002/002"), ("FF", "003/003")):
            base = os.path.join("workingData", "hamiltonian", "propagatorsL", path)
            ang["V_" + name] = np.stack([np.fromfile(os.path.join(base, f"V{m:03d}.bin")).reshape(N_L_ANG, N_L_ANG)
                                         for m in range(N_M)])
            ang["D_" + name] = np.stack([np.fromfile(os.path.join(base, f"D{m:03d}.bin")) for m in range(N_M)])
    finally:
        os.chdir(cwd)
        shutil.rmtree(work, ignore_errors=True)
    np.savez_compressed(OUT, n_r=N_R, n_l=N_L, n_m=N_M, n_l_ang=N_L_ANG, r_max=R_MAX, r_mask=R_MASK, zeta=ZETA,
                        dt=DT, r=r, drdx=drdx, T=np.real(T), P=P, cap=np.real(cap), v0=v0, vscf=vscf, W=W, **ang)
    print("wrote", OUT)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/src")
