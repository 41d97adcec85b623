"""The column kernel's RBL picks for every kind of pick stride, against the FP64 oracle.

The column kernel takes the picks -- every pice-th shell atom in traversal order
(RunWorklet.cpp:955-970) -- once per block of 32 steps from a shell mask: by exclusive prefix
parities when pice is a power of two (pick_shells_pow2), by walking the mask's bits otherwise, and
the count of shells still to skip carries across blocks, rows and tiles.  The saline stream only
has pice 4, so the sample count is varied here to give pice 1, 2, 3, 4, 5, 8 and 13, in the
reference's stride mode (first pick at rank 0) and the Philox offset mode (a per-atom first rank).
A pick that differs moves an atom's force by about 1e-3 of the force norm; mixed precision with the
exact classification stays within 1e-4 of the FP64 oracle.
"""
import os

import numpy as np
import pytest

from rbmd_b200 import _abi as A
from rbmd_b200 import synth

from conftest import rel_rms

pytestmark = pytest.mark.gpu

SAMPLES = {1: 400, 2: 200, 3: 130, 4: 100, 5: 80, 8: 50, 13: 30}


def _add_column(ctx_factory, sd):
    ctx = ctx_factory()
    old = os.environ.get("RBMD_PAIR_LAYOUT")
    os.environ["RBMD_PAIR_LAYOUT"] = "column"
    try:
        sid = ctx.add_system(sd)
    finally:
        if old is None:
            os.environ.pop("RBMD_PAIR_LAYOUT", None)
        else:
            os.environ["RBMD_PAIR_LAYOUT"] = old
    return ctx, sid


@pytest.mark.parametrize("mode", ["stride", "philox"])
@pytest.mark.parametrize("pice", sorted(SAMPLES))
def test_column_picks_against_oracle(ctx_factory, oracle_mod, pice, mode):
    sd = synth.saline(3000, seed=40 + pice)
    sd.params.neighbor_sample_num = SAMPLES[pice]
    sd.params.rbl_mode = A.RBL_STRIDE if mode == "stride" else A.RBL_PHILOX
    sd.params.precision = A.PREC_MIXED
    ctx, sid = _add_column(ctx_factory, sd)
    assert ctx.derived(sid)["pice_num"] == pice
    ctx.set_step(sid, 17)  # Philox offsets keyed by a step other than 0
    ctx.compute_forces(sid)
    ref = sd.copy()
    ref.params.precision = A.PREC_FP64
    o = oracle_mod.Oracle(ref)
    o.set_step(17)
    o.compute_forces()
    err = rel_rms(ctx.forces(sid), o.forces())
    assert err < 1e-4, err


@pytest.mark.parametrize("mode", ["stride", "philox"])
def test_column_atoms_outside_box(ctx_factory, oracle_mod, mode):
    """Atoms outside [lo, hi) -- one exactly on hi, one a whole box length past it, one below lo --
    are binned clamped but walk the neighbourhood of their unclamped cell; in the column layout the
    stray pass before the column kernel walks them (its own first pick in the Philox offset mode)
    and the column kernel adds their forces to the RBL mean.  Mixed precision against the FP64
    oracle, all atoms and the three one by one."""
    sd = synth.saline(3000, seed=61)
    L = sd.box_hi[0] - sd.box_lo[0]
    sd.pos = sd.pos.copy()
    sd.pos[0, 0] = sd.box_hi[0]
    sd.pos[7, 1] += L
    sd.pos[11, 2] = sd.box_lo[2] - 0.05
    sd.params.rbl_mode = A.RBL_STRIDE if mode == "stride" else A.RBL_PHILOX
    sd.params.precision = A.PREC_MIXED
    ctx, sid = _add_column(ctx_factory, sd)
    ctx.set_step(sid, 17)
    ctx.compute_forces(sid)
    f = ctx.forces(sid)
    ref = sd.copy()
    ref.params.precision = A.PREC_FP64
    o = oracle_mod.Oracle(ref)
    o.set_step(17)
    o.compute_forces()
    fo = o.forces()
    assert rel_rms(f, fo) < 1e-4, rel_rms(f, fo)
    for a in (0, 7, 11):
        assert np.linalg.norm(f[a] - fo[a]) < 1e-4 * np.linalg.norm(fo[a]) + 1e-6 * np.abs(fo).max(), a
    assert ctx.thermo(sid)["status"] == 0
