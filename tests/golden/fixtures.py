"""Loaders for the golden fixtures converted by make_golden.py."""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ["rpt02", "rpt09", "upt01", "upt03", "uft02"]


def load(name):
    z = np.load(os.path.join(HERE, name + ".npz"))
    case = {k: z[k] for k in z.files}
    for k in ("oa", "va", "ob", "vb"):
        case[k] = int(case[k])
    case["kind"] = str(case["kind"])
    case["e_ref"] = float(case["e_ref"])
    return case


def energies():
    with open(os.path.join(HERE, "energies.json")) as fp:
        return json.load(fp)


def reference_energy(case, mp=False):
    """The reference library (oracle/_ref) on a fixture.  Checker use only."""
    from oracle import oracle
    return oracle.solve(oracle.reference(), case, mp=mp)
