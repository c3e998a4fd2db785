"""Regenerate the golden fixtures of tests/golden (run from the repo root:
``python tests/golden/make_golden.py``).

The reference Fortran cannot run in this image, so the fixtures are outputs
of the CPU oracle (oracle/), itself pinned by the reference's known-answer
data (tests/test_oracle_known_answers.py).  Inputs are regenerated from the
documented seeded generator (duct_b200/synth.py); the fixture stores the
inputs' checksum so a generator change is caught.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from duct_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def cfg0():
    c = synth.config("cfg0")
    m, nm = c["my"], c["nmodes"]
    rhs = synth.chebyshev_rhs(m, m, nm, seed=0, ib=0)
    xalp = c["alp"] * np.arange(nm)
    alambda = c["fields"][0][2]
    ops = O.Ops(m)
    sol, _ = O.helm3d(rhs, ops, "d", alambda, xalp)
    np.savez(os.path.join(HERE, "cfg0_dirichlet.npz"), sol=sol, xalp=xalp, alambda=alambda,
             rhs_sum=np.array([rhs.real.sum(), rhs.imag.sum(), np.abs(rhs).sum()]))


def neumann_small():
    m, nm = 17, 5
    rhs = synth.chebyshev_rhs(m, m, nm, seed=7, ib=0)
    xalp = 1.0 * np.arange(nm)
    ops = O.Ops(m)
    sol, _ = O.helm3d(rhs, ops, "n", 0.0, xalp)
    np.savez(os.path.join(HERE, "neumann17.npz"), sol=sol, xalp=xalp, alambda=0.0,
             iofzero=ops.iofzero,
             rhs_sum=np.array([rhs.real.sum(), rhs.imag.sum(), np.abs(rhs).sum()]))


if __name__ == "__main__":
    cfg0()
    neumann_small()
    print(sorted(os.listdir(HERE)))
