"""Turn the reference binary's outputs into committed golden fixtures.

The reference ``main.cu`` is built for sm_100a from its own sources by ``oracle/build_ref.py``
and run on a B200 by ``oracle/run_ref.sh <dir>``; this script reads ``<dir>/<case>/`` (the
reference's ``output/`` tree and ``case.json``) and writes ``tests/golden/ref_<case>.npz`` with

    dipole   complex128 [N_l][N_kso][N_t]  the dipL%03d.bin files (h_writeDipoleMoment.cuh:1-23)
    E        float64 [N_t]                  the E%03d.bin file the run used (h_writeField)
    case     JSON text: the input-generator arguments (problems.reference_like) of the case

Usage:  python tests/golden/make_ref_fixtures.py <dir>   (the directory oracle/run_ref.sh wrote)
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from ggbtddft_b200 import workingdata as WD  # noqa: E402


def main(src):
    for case in sorted(os.listdir(src)):
        cj_path = os.path.join(src, case, "case.json")
        if not os.path.exists(cj_path):
            continue
        cj = json.load(open(cj_path))
        root = os.path.join(src, case, "output")
        dip = WD.read_dipole_outputs(root, cj["sim_date"], cj["sim_index"], 0, cj["n_kso"], cj["n_l"])
        E = np.fromfile(os.path.join(root, f"{cj['sim_date']:08d}", f"{cj['sim_index']:05d}",
                                     "timeDependent/field/E000.bin"))
        out = os.path.join(HERE, f"ref_{case}.npz")
        np.savez_compressed(out, dipole=dip, E=E, case=json.dumps(cj))
        print("wrote", out, dip.shape)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_ref_fixtures.py <dir written by oracle/run_ref.sh>")
    main(sys.argv[1])
