"""Build the reference's own ``main.cu`` for sm_100a on small parity configurations.

TEST INFRASTRUCTURE ONLY (the checker's checker): it produces ``oracle/_ref/<case>/`` with

    ggb_ref           the reference binary, compiled by nvcc from the reference's sources where they
                      lie (main.cu and subFunctions/ are symlinked, never copied) together with a
                      generated params.cuh for the case (sizes are compile-time in the reference)
    run/workingData/  the inputs in the reference's file layout
    output/           the (empty) directory tree the reference writes into
    case.json         the generator parameters, so tests can rebuild identical inputs

Run the binary on a GPU with ``cd oracle/_ref/<case>/run && ../ggb_ref``; it reads
``./workingData`` and writes ``../output/<date>/<idx>/...``.  ``tests/golden/make_ref_fixtures.py``
turns those outputs into the committed golden fixtures.

Timed cases (``TIMED_CASES``) are built the same way, with one addition in their generated
params.cuh: the reference's ``h_timePropagation`` (h_timePropagation.cuh:32-114) is included under
another name and wrapped by a function of that name that brackets it with cudaEvents and prints
``GGB_REF_TIMING scan=<s> steps=<N_t> ms=<t>`` (the reference's sources are not modified; main.cu
calls the wrapper).  Their workingData is large (W alone is N_l N_r^2 16 bytes), so it is not
written here: ``oracle/time_ref.py`` writes it on the GPU machine and runs the binary.

The reference's GSL includes are unused (main.cu:15-18); empty stub headers satisfy them.
``-arch=sm_30`` of ``src/compile:1`` is not supported by CUDA 12.9, so the build targets sm_100a.
Only sizes that are multiples of 32 are valid for the reference (its launch grids truncate).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, REPO)

REF_SRC = "/root/reference/src"
OUT = os.path.join(HERE, "_ref")
SIM_DATE, SIM_INDEX = 20000101, 0

# case name -> reference_like() keyword arguments
CASES = {
    "h64": dict(n_r=64, n_l=32, n_t=128, atom="H", r_mask=30.0, zeta_ref=1.0, dt_as=20.0,
                intensity=2e14, omega0=0.057, cycles=1.0),
    "ne3_64": dict(n_r=64, n_l=32, n_t=64, atom="Ne3", r_mask=20.0, zeta_ref=1.0, dt_as=10.0,
                   intensity=3e14, omega0=0.057, cycles=1.0, perturb=0.05, seed=7),
    # twice the radial and angular sizes, every coupling and the Hartree/exchange phases active
    "ne3_128": dict(n_r=128, n_l=64, n_t=48, atom="Ne3", r_mask=30.0, zeta_ref=1.0, dt_as=10.0,
                    intensity=3e14, omega0=0.057, cycles=1.0, perturb=0.05, seed=11),
    # all-electron argon (nine orbitals, m = 0 and 1), every coupling active
    "ar9_256": dict(n_r=256, n_l=64, n_t=32, atom="Ar9", r_mask=60.0, zeta_ref=2.0 * 0.5 / 90.0,
                    dt_as=0.02 / 0.041341373335182, intensity=1.4e14, omega0=0.057, cycles=1.0),
}


# timed case name -> reference_like() keyword arguments (sizes multiples of 32, as the reference needs)
TIMED_CASES = {
    "ar9_608": dict(n_r=608, n_l=96, n_t=200, atom="Ar9", r_mask=200.0, zeta_ref=2.0 * 0.5 / 300.0,
                    dt_as=0.02 / 0.041341373335182,
                    intensity=1.4e14, omega0=0.057, cycles=2.0),
}

TIMING_WRAPPER = """
// Timing wrapper of this build only (not part of the reference): the reference's h_timePropagation
// is included above under the name h_timePropagation_untimed and bracketed here by cudaEvents.
void h_timePropagation (ksoSetTDStruct ksoSetTD, hartreeStruct hartree, propagatorsStruct propagators,
                        meshStruct mesh, observableStruct observables, tempStruct temp, handleStruct handles,
                        int scandx)
{
	cudaEvent_t ggb_e0, ggb_e1;
	float ggb_ms = 0.0f;
	cudaEventCreate(&ggb_e0);
	cudaEventCreate(&ggb_e1);
	cudaDeviceSynchronize();
	cudaEventRecord(ggb_e0, 0);
	h_timePropagation_untimed(ksoSetTD, hartree, propagators, mesh, observables, temp, handles, scandx);
	cudaEventRecord(ggb_e1, 0);
	cudaEventSynchronize(ggb_e1);
	cudaEventElapsedTime(&ggb_ms, ggb_e0, ggb_e1);
	printf("GGB_REF_TIMING scan=%d steps=%d ms=%.4f\\n", scandx, N_t, ggb_ms);
	cudaEventDestroy(ggb_e0);
	cudaEventDestroy(ggb_e1);
}
"""


def add_timing_wrapper(params_path: str) -> None:
    """Rename the reference's h_timePropagation at its include and append the timed wrapper."""
    inc = '#include "./subFunctions/timePropagation/h_timePropagation.cuh"'
    s = open(params_path).read()
    assert s.count(inc) == 1
    s = s.replace(inc, "#define h_timePropagation h_timePropagation_untimed\n" + inc + "\n#undef h_timePropagation")
    with open(params_path, "w") as f:
        f.write(s + TIMING_WRAPPER)


def field_params(kw):
    import math
    from ggbtddft_b200 import inputs as I
    omega0 = kw.get("omega0", 0.057)
    return dict(e0=I.intensity_to_e0(kw.get("intensity", 2e14)), omega0=omega0,
                tau0=kw.get("cycles", 1.0) * 2.0 * math.pi / omega0, cep0=kw.get("cep", 0.5 * math.pi))


def build_case(name: str, kw: dict, nvcc: str = "nvcc", timed: bool = False) -> str:
    from ggbtddft_b200 import problems as P, workingdata as WD
    d = os.path.join(OUT, name)
    os.makedirs(os.path.join(d, "run"), exist_ok=True)
    run = P.reference_like(**kw)
    fp = field_params(kw)
    Z = {"H": 1.0, "Ne3": 8.0, "Ar9": 18.0}[kw.get("atom", "H")]
    if not timed:
        WD.write_working_data(run, os.path.join(d, "run"))
    WD.write_params_cuh(run, os.path.join(d, "params.cuh"), sim_date=SIM_DATE, sim_index=SIM_INDEX, Z=Z, **fp)
    if timed:
        add_timing_wrapper(os.path.join(d, "params.cuh"))
    WD.output_dirs(os.path.join(d, "output"), SIM_DATE, SIM_INDEX, 1, run.n_orb)
    for link, target in (("main.cu", f"{REF_SRC}/main.cu"), ("subFunctions", f"{REF_SRC}/subFunctions")):
        p = os.path.join(d, link)
        if os.path.lexists(p):
            os.remove(p)
        os.symlink(target, p)
    stub = os.path.join(OUT, "gslstub", "gsl")
    os.makedirs(stub, exist_ok=True)
    for h in ("gsl_sf_laguerre", "gsl_sf_legendre", "gsl_sf_coulomb", "gsl_sf_fermi_dirac"):
        open(os.path.join(stub, h + ".h"), "a").close()
    cmd = [nvcc, "main.cu", "-I", os.path.join(OUT, "gslstub"), "-O2",
           "-gencode", "arch=compute_100a,code=sm_100a", "-lcublas", "-lcusolver", "-lcufft", "-o", "ggb_ref"]
    try:
        subprocess.run(cmd, cwd=d, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    finally:
        # the links are only needed by the compiler; removing them keeps copies of this folder
        # (e.g. to a GPU machine) from following them into the reference tree
        for link in ("main.cu", "subFunctions"):
            os.remove(os.path.join(d, link))
    with open(os.path.join(d, "case.json"), "w") as f:
        json.dump(dict(name=name, kwargs=kw, field=fp, sim_date=SIM_DATE, sim_index=SIM_INDEX,
                       n_l=run.n_l, n_kso=run.n_orb, n_t=run.n_t, n_r=run.n_r), f, indent=1)
    return d


def main(argv=None):
    if not os.path.isdir(REF_SRC):
        print("reference sources not present; nothing to build")
        return 0
    names = (argv or sys.argv[1:]) or list(CASES) + list(TIMED_CASES)
    for n in names:
        if n in TIMED_CASES:
            print("built", build_case(n, TIMED_CASES[n], timed=True))
        else:
            print("built", build_case(n, CASES[n]))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
