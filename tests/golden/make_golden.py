"""Builds the committed golden fixtures from the reference's own example files.

Usage: python make_golden.py <path to the gpu-tild sources>.  Only a checkout that has those
sources runs it; the GPU box never needs them.  Outputs, next to this script:
  coacervate_config.npz   examples/Coacervate/input.data parsed as read_charge_config does
                          (positions FP32 via %f, types, charges, bond list)
  coacervate_step0.json   the step-0 line of examples/Coacervate/data.dat, the input script
                          examples/Coacervate/input and the runtime-parameter echo
                          examples/Coacervate/NEED_A_NAME.input (the known-answer tests)
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(HERE, "..", "..", "gpu-tild_b200")]
import tild_systems as ts  # noqa: E402

def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: python make_golden.py <path to the gpu-tild sources>")
    REF = sys.argv[1]
    ex = os.path.join(REF, "examples", "Coacervate")
    d = ts.read_data_file(os.path.join(ex, "input.data"), 3, True)
    np.savez_compressed(os.path.join(HERE, "coacervate_config.npz"), x=d["x"], types=d["types"].astype(np.int8),
                        mol=d["mol"], charges=d["charges"].astype(np.int8), bonds=d["bonds"].astype(np.int32),
                        box=np.array(d["box"], np.float32), mass=np.array(d["mass"], np.float32))
    header, line = open(os.path.join(ex, "data.dat")).read().strip().split("\n")[:2]
    vals = [float(v) for v in line.split()]
    script = open(os.path.join(ex, "input")).read()
    gold = {
        "source": "examples/Coacervate/data.dat line 2 (step 0) and examples/Coacervate/input",
        "header": header.strip(),
        "step": int(vals[0]), "Upe": vals[1], "Ubond": vals[2], "P": vals[3:9], "Ugauss": vals[9:],
        "script": {"Dim": 3, "Nx": [21, 21, 225], "pmeorder": 1, "charges": [0.43484, 1.0],
                   "gaussian": [[1, 1, 0.0003688, 1.0]], "bond": [1.5, 0.0], "delt": 0.005},
        "script_text": script,
        "need_a_name_input": open(os.path.join(ex, "NEED_A_NAME.input")).read(),
    }
    with open(os.path.join(HERE, "coacervate_step0.json"), "w") as f:
        json.dump(gold, f, indent=1)


if __name__ == "__main__":
    main()
