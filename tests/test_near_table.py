"""The reference's near-Coulomb lookup table (RBMD_NEAR_TABLE), on the CPU.

The reference evaluates the RBL near Coulomb force with G(r) read from a table built for
alpha = 0.1 (staticTable/ExecStaticTable.h:96-135, model/ERFTable.h): the key of a distance is
bits 15-25 of its FP32 pattern (the exponent's low three bits over the mantissa's top eight), no
interpolation.  Checked here: the library's key and table against the oracle's (written
separately), the table's grid points, and -- where the reference tree is present -- every row of
the reference's own table files (res/json_files/Gnear_table_leq2_2.txt, Gnear_table_geq2_2.txt).
"""
import ctypes as C
import math
import os
import struct

import numpy as np
import pytest

from rbmd_b200 import _abi as A

import refinputs as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "rbmd_b200", "_lib", "librbmd_b200.so")
FILES = {"leq2_2": "res/json_files/Gnear_table_leq2_2.txt", "geq2_2": "res/json_files/Gnear_table_geq2_2.txt"}


@pytest.fixture(scope="module")
def lib():
    L = C.CDLL(LIB)
    A.declare(L)
    return L


def lib_table(L):
    out = np.zeros(2048, np.float32)
    assert L.rbmd_near_table_default(out.ctypes.data_as(C.POINTER(C.c_float))) == A.OK
    return out


def py_key(r):
    (bits,) = struct.unpack("<I", struct.pack("<f", r))
    return (bits & (2 ** 26 - 2 ** 15)) >> 15


def g_alpha01(r):
    a = 0.1
    return math.erfc(math.sqrt(a) * r) / (r * r) + 2 * math.sqrt(a) * math.exp(-a * r * r) / (math.sqrt(math.pi) * r)


def test_key_of_a_distance(lib, oracle_mod):
    rng = np.random.default_rng(3)
    rs = np.concatenate([rng.uniform(0.1, 12.0, 4000), [0.1, 0.1001, 1.9961, 2.0, 2.008, 11.969, 11.999]])
    for r in rs.astype(np.float32):
        k = py_key(float(r))
        assert lib.rbmd_near_table_key(float(r)) == k == oracle_mod.near_key(float(r))
    # the reference's ranges: [0.1, 2) -> 921..2047, [2, 12) -> 0..639
    assert py_key(0.1) == 921 and py_key(np.nextafter(np.float32(2.0), np.float32(0.0))) == 2047
    assert py_key(2.0) == 0 and py_key(np.nextafter(np.float32(12.0), np.float32(0.0))) == 639


def test_library_table_equals_oracle(lib, oracle_mod):
    assert np.array_equal(lib_table(lib), oracle_mod.near_table())


def test_table_points(lib):
    """Each key holds G at the first point of the reference's walk (0.1 + 0.0001 m below 2,
    2 + 0.001 m below 12) that has the key; keys outside the walks hold G at their lower edge."""
    tab = lib_table(lib)
    seen = {}
    for r0, dr, r1 in ((0.1, 1e-4, 2.0), (2.0, 1e-3, 12.0)):
        m = 0
        while r0 + m * dr < r1:
            r = r0 + m * dr
            seen.setdefault(py_key(r), r)
            m += 1
    assert sorted(seen) == list(range(0, 640)) + list(range(921, 2048))
    for k, r in seen.items():
        assert tab[k] == np.float32(g_alpha01(r)), (k, r)
    for k in list(range(640, 921)):
        e3 = k >> 8
        edge = math.ldexp(1 + (k & 255) / 256, 1 + e3 if e3 <= 2 else e3 - 7)
        assert tab[k] == np.float32(g_alpha01(edge)), k


@pytest.mark.skipif(not R.available(), reason="reference tree not present")
@pytest.mark.parametrize("name", sorted(FILES))
def test_table_pinned_to_reference_files(lib, name):
    """Every row of the reference's table: its key is that of its distance, and its G (printed to
    six digits) is the library's to the printing precision below r = 8; beyond, the files' values
    drift from the FP64 G, to 1% at r = 12 (as 1 - erf taken in single precision would), so there
    within 1.1% (G is below 1e-3 of G(2) there)."""
    tab = lib_table(lib)
    rows = [ln.split() for ln in open(os.path.join(R.REF_ROOT, FILES[name])) if ln.strip()]
    assert len(rows) == {"leq2_2": 1127, "geq2_2": 640}[name]
    keys = np.array([int(r[0]) for r in rows])
    dist = np.array([float(r[1]) for r in rows])
    g = np.array([float(r[3]) for r in rows])
    assert all(py_key(d) == k for d, k in zip(dist, keys))
    assert np.array_equal(keys, np.arange(921, 2048) if name == "leq2_2" else np.arange(0, 640))
    rel = np.abs(tab[keys].astype(np.float64) - g) / np.abs(g)
    near = dist < 8.0
    assert rel[near].max() < 6e-6, rel[near].max()
    assert rel.max() < 1.1e-2, rel.max()


@pytest.mark.skipif(not R.available(), reason="reference tree not present")
def test_host_reads_reference_table_files(tmp_path):
    """coulomb.near_table given as the two files: the resolved system carries their G by key."""
    path, _ = R.resolve(R.INPUTS["lj_salt_box"], tmp_path)
    import json
    import re
    text = open(path).read()
    files = [os.path.join(R.REF_ROOT, FILES[k]) for k in ("leq2_2", "geq2_2")]
    text, n = re.subn(r'("coulomb"\s*:\s*\{)', r'\g<1> "near_table": %s,' % json.dumps(files), text, count=1)
    assert n == 1
    open(path, "w").write(text)
    r, j = R.dump(path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert j["params"]["near_table"] == A.NEAR_TABLE
    tab = np.asarray(j["near_table_values"], np.float32)
    for k in ("leq2_2", "geq2_2"):
        for row in (ln.split() for ln in open(os.path.join(R.REF_ROOT, FILES[k])) if ln.strip()):
            assert tab[int(row[0])] == np.float32(float(row[3]))
