"""The oracle's real-space Coulomb kernel G(r) against the reference's own alpha = 0.1 tables
(res/json_files/Gnear_table_{leq2,geq2}_2.txt, compiled into framework/model/ERFTable.h and
indexed by FP32 bits in staticTable/ExecStaticTable.h:96-135).

Column 4 is G(r) = erfc(sqrt(a) r) / r^2 + 2 sqrt(a) exp(-a r^2) / (sqrt(pi) r); the oracle's near
force on isolated pairs reproduces it at every tabulated r to the tables' printed precision (see
gnear_pairs.table_tolerance).  Column 5 is the tables' linear-interpolation slope
(`erf_gnear_der_*`), read only by the interpolation that ExecStaticTable::TableGnearValue has
commented out (:111-118), so it never reaches a force; below r = 0.5 it is dG/dr (checked against
the oracle's finite difference), beyond it drifts from dG/dr by up to 16%.
The committed fixture tests/golden/gnear_alpha0.1.txt (every third row) is checked everywhere; the
full tables where the reference tree is present.
"""
import os

import numpy as np
import pytest

import gnear_pairs as GP
import refinputs

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "gnear_alpha0.1.txt")


def oracle_g(oracle_mod, rs):
    o = oracle_mod.Oracle(GP.system(rs))
    o.compute_forces()
    near = o.force_part(0)
    return near[0::2, 0], near[1::2, 0]


def test_fixture_rows(oracle_mod):
    r, g, _ = GP.table(FIXTURE)
    assert len(r) > 500 and r.min() == pytest.approx(0.1) and r.max() > 11.9
    gi, gj = oracle_g(oracle_mod, r)
    assert np.allclose(gj, -gi, rtol=0, atol=0)  # equal and opposite, exactly
    bad = np.abs(gi - g) > GP.table_tolerance(r, g)
    assert not bad.any(), list(zip(r[bad][:5], gi[bad][:5], g[bad][:5]))


@pytest.mark.skipif(not refinputs.available(), reason="reference tree not present")
def test_full_reference_tables(oracle_mod):
    r, g, s = GP.reference_tables(refinputs.REF_ROOT)
    assert len(r) == 1127 + 640
    gi, _ = oracle_g(oracle_mod, r)
    bad = np.abs(gi - g) > GP.table_tolerance(r, g)
    assert not bad.any(), list(zip(r[bad][:5], gi[bad][:5], g[bad][:5]))
    # the fixture is a faithful subset
    fr, fg, fs = GP.table(FIXTURE)
    idx = np.searchsorted(r[:1127], fr[fr < 2.0])
    assert np.array_equal(r[:1127][idx], fr[fr < 2.0]) and np.array_equal(g[:1127][idx], fg[fr < 2.0])


def test_slope_column_is_dgdr_at_short_range(oracle_mod):
    r, _, s = GP.table(FIXTURE)
    sel = r < 0.5
    r, s = r[sel], s[sel]
    h = 1e-5 * r
    gp, _ = oracle_g(oracle_mod, r + h)
    gm, _ = oracle_g(oracle_mod, r - h)
    d = (gp - gm) / (2 * h)
    assert np.all(np.abs(d / s - 1) < 5e-3)
