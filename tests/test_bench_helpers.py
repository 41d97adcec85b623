"""bench.py's measurement helpers that need no GPU: the reciprocal-space Ewald force used as the
denominator of the k-space-only RBE error (against the oracle's far force), the converged kmax,
and the serving stream's size strata behind the CPU baselines."""
import os
import sys

import numpy as np
import pytest

from rbmd_b200 import _abi as A
from rbmd_b200 import synth

from conftest import rel_rms

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_ewald_kspace_matches_oracle_far_force(oracle_mod):
    sd = synth.nacl_melt(n_side=6, coulomb=A.COUL_EWALD, kmax=(5, 5, 5), precision=A.PREC_FP64)
    rng = np.random.default_rng(3)
    sd.pos = np.ascontiguousarray((sd.pos + rng.normal(scale=0.1, size=sd.pos.shape)) % sd.box_hi[0])
    o = oracle_mod.Oracle(sd)
    o.compute_forces()
    f = bench.ewald_kspace_forces(sd.pos, sd.charge, sd.box_hi - sd.box_lo, sd.params.alpha, (5, 5, 5))
    assert rel_rms(f, o.force_part(1)) < 1e-10


def test_converged_kmax():
    km = bench.converged_kmax([21.7, 21.7, 30.0], 0.09)
    kc = np.sqrt(-4 * 0.09 * np.log(1e-12))
    assert km[0] == int(np.ceil(kc * 21.7 / (2 * np.pi))) and km[2] > km[0]
    k = 2 * np.pi * km[0] / 21.7
    assert np.exp(-k * k / (4 * 0.09)) < 1e-12


def test_stream_strata_cover_the_stream():
    st = bench.stream_strata(512)
    sizes, _ = synth.serving_stream(n_requests=512)
    assert sum(s["requests"] for s in st) == 512 and sum(s["atoms"] for s in st) == int(sizes.sum())
    for s in st:
        assert s["lo"] <= s["size"] < s["hi"]


def test_profiled_figures_of_the_column_kernel():
    """The roofline fields that the bench line takes from the committed ncu summary of the column
    kernel: all three present, and the DRAM traffic at least the algorithmic 64 B per atom."""
    fig = bench.profiled_figures("pair_col")
    assert fig["source"] == "profiles/k_pair_col_saline_small.md"
    assert fig["traffic_bytes_per_atom"] >= 64.0
    assert 0.0 < fig["issue_active_pct"] <= 100.0
    assert fig["warp_inst_per_atom"] > 0.0


def test_reference_arm_line():
    """`bench.py --impl reference` on a tiny CPU sample: one JSON line with the reference arm's
    keys -- the oracle port's throughput, its cpu_baseline and an e2e without device copies."""
    import json
    import subprocess
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--cpu-seconds", "0.5"], capture_output=True, text=True, timeout=600,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference" and d["unit"] == bench.UNIT and d["metric"] == bench.METRIC
    assert d["value"] > 0 and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"] and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
