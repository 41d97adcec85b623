"""Energies along a run against the FP64 oracle's, not only against the GPU's own FP64 path.

C1's LJ fluid (4000 atoms from fcc, RBL with 100 shell samples, NVE, dt 0.005), 500 steps: the total
energy every 50 steps on the GPU in FP64 and in mixed precision, and in the FP64 oracle over the
same run.  Perturbing the start by 1e-12 moves the oracle's own energies by under 1e-12 of |E_0|
over these 500 steps, so the FP64 GPU path is held to 1e-8; the mixed path (forces within 1e-5 of
FP64) to 5e-4, the size of its measured drift difference over 1000 steps.  The saline system
(RBE + RBL, SHAKE, NVT) is checked the same way over 100 steps in FP64, to 1e-6: SHAKE iterates to
a relative tolerance of 1e-5, so a triple may take one iteration more on one side.
"""
import numpy as np
import pytest

from rbmd_b200 import _abi as A
from rbmd_b200 import synth

pytestmark = pytest.mark.gpu


def _energies(run, nsamples, every):
    e = [run(0)]
    for _ in range(nsamples):
        e.append(run(every))
    return np.array(e)


def _gpu(ctx_factory, sd, nsamples, every):
    ctx = ctx_factory(graphs=True)
    sid = ctx.add_system(sd)
    ctx.init(sid)

    def run(k):
        if k:
            ctx.step(sid, k)
        th = ctx.thermo(sid)
        assert th["status"] == 0
        return th["total_energy"]
    return _energies(run, nsamples, every)


def _oracle(oracle_mod, sd, nsamples, every):
    ref = sd.copy()
    ref.params.precision = A.PREC_FP64
    o = oracle_mod.Oracle(ref)
    o.init()

    def run(k):
        if k:
            o.step(k)
        return o.thermo()["total_energy"]
    return _energies(run, nsamples, every)


@pytest.fixture(scope="module")
def lj_oracle(oracle_mod):
    return _oracle(oracle_mod, synth.lj_fcc(), 10, 50)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_lj_nve_energy_tracks_oracle(ctx_factory, lj_oracle, prec):
    sd = synth.lj_fcc(precision=A.PREC_FP64 if prec == "fp64" else A.PREC_MIXED)
    e = _gpu(ctx_factory, sd, 10, 50)
    eo = lj_oracle
    e0 = abs(eo[0])
    diff = np.abs(e - eo) / e0
    drift, drift_o = (e[-1] - e[0]) / e0, (eo[-1] - eo[0]) / e0
    if prec == "fp64":
        assert diff.max() < 1e-8, diff
    else:
        assert diff.max() < 5e-4, diff
        assert abs(drift - drift_o) < 5e-4, (drift, drift_o)


def test_saline_energy_tracks_oracle(ctx_factory, oracle_mod):
    sd = synth.saline(2000, seed=8)
    sd.params.precision = A.PREC_FP64
    e = _gpu(ctx_factory, sd, 4, 25)
    eo = _oracle(oracle_mod, sd, 4, 25)
    diff = np.abs(e - eo) / abs(eo[0])
    assert diff.max() < 1e-6, diff
