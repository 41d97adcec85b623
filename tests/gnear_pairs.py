"""Isolated charge pairs at chosen distances, for reading the real-space Coulomb kernel G(r) off
the near force.

Pair k puts a +1 charge at a lattice site and a -1 charge r_k further along x; sites are 26 apart,
so with rc = 12.5 every atom sees its partner only.  LJ is off (epsilon 0), units LJ (qqr2e 1),
alpha 0.1, Verlet neighbours (every pair within rc), Ewald with kmax 1 for the far part.  The near
force on the +1 atom is -q_i q_j G(r) (r_j - r_i) / r = G(r) along +x
(RunWorklet.cpp:2890-2985, ExecForceFunction.h Gnear:682-689).
"""
import math

import numpy as np

from rbmd_b200 import _abi as A
from rbmd_b200 import synth

SPACING = 26.0
ALPHA = 0.1
RC = 12.5


def table(path):
    r, g, s = [], [], []
    for ln in open(path):
        if ln.startswith("#") or not ln.strip():
            continue
        w = ln.split()
        r.append(float(w[0]))
        g.append(float(w[1]))
        s.append(float(w[2]))
    return np.array(r), np.array(g), np.array(s)


def reference_tables(root):
    rows = []
    for name in ("Gnear_table_leq2_2.txt", "Gnear_table_geq2_2.txt"):
        for ln in open(f"{root}/res/json_files/{name}"):
            w = ln.split()
            if len(w) == 5:
                rows.append([float(w[1]), float(w[3]), float(w[4])])
    a = np.array(rows)
    return a[:, 0], a[:, 1], a[:, 2]


def system(rs, precision=A.PREC_FP64):
    rs = np.asarray(rs, np.float64)
    n = len(rs)
    side = int(math.ceil(n ** (1.0 / 3.0) - 1e-9))
    L = side * SPACING
    k = np.arange(n)
    site = np.stack([k % side, (k // side) % side, k // (side * side)], 1) * SPACING + 1.0
    pos = np.empty((2 * n, 3))
    pos[0::2] = site
    pos[1::2] = site
    pos[1::2, 0] += rs
    charge = np.empty(2 * n)
    charge[0::2], charge[1::2] = 1.0, -1.0
    params = A.default_params(force_field=A.FF_LJ_CUT_COUL_LONG, neighbor=A.NEIGH_VERLET, cut_off=RC, r_core=RC,
                              coulomb=A.COUL_EWALD, alpha=ALPHA, kmax=(1, 1, 1), units=A.UNITS_LJ,
                              timestep=0.001, temp_ctrl=A.TC_NONE, ensemble=A.ENS_NVE, precision=precision)
    return synth.SystemData(pos, np.ones(2 * n), np.zeros(2 * n), [0.0], [1.0], [0, 0, 0], [L, L, L],
                            vel=np.zeros((2 * n, 3)), charge=charge, params=params, name=f"gnear_pairs_{n}")


def table_tolerance(r, g):
    """The printed tables carry six significant digits and were computed in single precision with
    erfc formed as 1 - erf (the large-r rows lose digits to that cancellation): one FP32 unit of
    1 - erf near 1, divided by r^2, on top of the print rounding."""
    return 6e-6 * np.abs(g) + 2.0 ** -23 / (r * r) + 1e-14
