"""Pair kernels that cull cells geometrically, after SHAKE moved atoms.

The reference builds the cell list before the water constraint (ExecutionNVT.cpp:78-119,
843-870) and its SHAKE wraps a constrained atom that it moves out of the box back in
(MolecularWorklet.h:2585-2610); the force evaluation then visits each atom in its old cell, at the
wrapped position.  The lean and column kernels skip cells that cannot hold an atom within rc; they
must widen that test by the distance SHAKE moved atoms and keep the cells of atoms it wrapped.
A water box whose bonds start 25% too long makes SHAKE move atoms by tenths of an angstrom (and
wrap some of them) in the first step; the culling layouts must then give the forces of the layouts
that walk every stencil cell (general in FP64, tile in mixed precision).
"""
import os

import numpy as np
import pytest

from rbmd_b200 import _abi as A
from rbmd_b200 import synth

pytestmark = pytest.mark.gpu


def _stretched_water(precision):
    sd = synth.spce_water(n_mol=1000, precision=precision, temp_ctrl=A.TC_BERENDSEN,
                          temperature=(300.0, 300.0, 100.0))
    L = sd.box_hi - sd.box_lo
    b = sd.bond_atoms.reshape(-1, 2)
    o, h = b[:, 0], b[:, 1]
    d = sd.pos[h] - sd.pos[o]
    d -= L * np.round(d / L)
    pos = sd.pos.copy()
    pos[h] = pos[o] + 1.25 * d
    # shift so that many molecules straddle the faces, then wrap
    sd.pos = np.ascontiguousarray((pos + 0.37 * (L / 6.0) - sd.box_lo) % L + sd.box_lo)
    return sd


def _forces_after(ctx_factory, sd, layout, steps):
    old = os.environ.get("RBMD_PAIR_LAYOUT")
    os.environ["RBMD_PAIR_LAYOUT"] = layout
    try:
        ctx = ctx_factory(graphs=False)
        sid = ctx.add_system(sd)
    finally:
        if old is None:
            os.environ.pop("RBMD_PAIR_LAYOUT", None)
        else:
            os.environ["RBMD_PAIR_LAYOUT"] = old
    ctx.init(sid)
    out = []
    for _ in range(steps):
        ctx.step(sid, 1)
        out.append(ctx.forces(sid))
    assert ctx.thermo(sid)["status"] == 0
    return out


def _per_atom_rel(f, g):
    return np.linalg.norm(f - g, axis=1) / np.maximum(np.linalg.norm(g, axis=1), 1e-3 * np.abs(g).max())


def test_lean_after_shake_equals_general_fp64(ctx_factory):
    sd = _stretched_water(A.PREC_FP64)
    ref = _forces_after(ctx_factory, sd, "atom", 3)
    got = _forces_after(ctx_factory, sd, "lean", 3)
    for f, g in zip(got, ref):
        assert _per_atom_rel(f, g).max() < 1e-9


def test_column_after_shake_equals_tile_mixed(ctx_factory):
    sd = _stretched_water(A.PREC_MIXED)
    ref = _forces_after(ctx_factory, sd, "cell", 3)
    got = _forces_after(ctx_factory, sd, "column", 3)
    for f, g in zip(got, ref):
        # FP32 sums in another order: ~1e-6; a pair missed or picked differently: 1e-2 and more
        assert _per_atom_rel(f, g).max() < 1e-3
