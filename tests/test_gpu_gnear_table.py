"""The FP64 GPU path's real-space Coulomb kernel G(r) against the reference's alpha = 0.1 table
(the committed every-third-row fixture of res/json_files/Gnear_table_{leq2,geq2}_2.txt): isolated
charge pairs (gnear_pairs), near force = the GPU's total force minus the oracle's Ewald far part."""
import os

import numpy as np
import pytest

import gnear_pairs as GP

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "gnear_alpha0.1.txt")


def test_gpu_g_matches_reference_table(ctx_factory, oracle_mod):
    r, g, _ = GP.table(FIXTURE)
    sd = GP.system(r)
    ctx = ctx_factory()
    sid = ctx.add_system(sd)
    ctx.compute_forces(sid)
    f = ctx.forces(sid)
    o = oracle_mod.Oracle(sd)
    o.compute_forces()
    near = f - o.force_part(1)  # the Ewald far part (kmax 1), identical arithmetic on both sides
    gi = near[0::2, 0]
    assert np.allclose(near[1::2, 0], -gi, rtol=1e-12, atol=1e-15)
    bad = np.abs(gi - g) > GP.table_tolerance(r, g)
    assert not bad.any(), list(zip(r[bad][:5], gi[bad][:5], g[bad][:5]))
    # and the GPU near force equals the oracle's at FP64 level
    assert np.allclose(gi, o.force_part(0)[0::2, 0], rtol=1e-12, atol=1e-16)
