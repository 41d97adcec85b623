"""Synthetic workload builders (CPU)."""
import numpy as np

from rbmd_b200 import synth


def test_water_special_lists_match_generic_builder():
    sd = synth.saline(3000, seed=4)
    nw = len(sd.angle_atoms) // 3
    bonds = sd.bond_atoms.reshape(-1, 2).tolist()
    off, ids, ws = synth.special_lists(sd.n, bonds, (0.0, 0.0, 0.0))
    assert np.array_equal(off, sd.special_offsets)
    assert np.array_equal(ids, sd.special_ids)
    assert np.array_equal(ws, sd.special_weights)
    assert sd.n - 3 * nw > 0  # ions present


def test_saline_composition_and_geometry():
    sd = synth.saline(20000, seed=9)
    assert abs(sd.n - 20000) < 60
    q = sd.charge
    assert abs(q.sum()) < 1e-9
    L = sd.box_hi[0]
    tri = sd.angle_atoms.reshape(-1, 3)
    d = sd.pos[tri[:, 0]] - sd.pos[tri[:, 1]]
    d -= L * np.round(d / L)
    assert np.allclose(np.sqrt((d * d).sum(1)), 1.0)
    dens = (sd.mass.sum() / 6.02214076e23) / (L * 1e-8) ** 3
    assert abs(dens - 1.0) < 0.02


def test_serving_stream_shape():
    sizes, arrivals = synth.serving_stream()
    assert len(sizes) == 512 and sizes.min() >= 1000 and sizes.max() <= 64000
    assert np.all(np.diff(arrivals) >= 0)
    assert 6.0 < arrivals[-1] < 15.0  # ~512 / 50 per s
