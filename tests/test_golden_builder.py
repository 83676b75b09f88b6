"""Bit-exact pins against outputs of the reference's own numpy code.

tests/golden/builder_small.npz was written by tests/golden/make_golden.py,
which imports the reference's ConstraintBuilderMixin
(src/muscle/constraint/builder.py), fix_tet_winding
(src/muscle/util/mesh_utils.py:16-32), RampActivationSource
(src/muscle/util/activation.py:28-44) and ConstraintType (src/muscle/defs.py)
and runs them on a 74-tet mesh with both windings and two degenerate tets.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from rlmusclev2_b200 import builder
from rlmusclev2_b200.defs import ConstraintType
from rlmusclev2_b200.meshgen import fix_tet_winding, ramp_activation

G = np.load(Path(__file__).parent / "golden" / "builder_small.npz")


def test_constraint_type_values():
    names = [str(n) for n in G["ctype_names"]]
    assert names == [m.name for m in ConstraintType]
    np.testing.assert_array_equal(G["ctype_values"], [int(m.value) for m in ConstraintType])


def test_rest_matrices_bit_exact():
    """_batch_compute_tet_rest_matrices (builder.py:28-43)."""
    B, V, valid = builder.tet_rest_data(G["pos0"], G["tets"])
    np.testing.assert_array_equal(valid, G["rest_valid"])
    np.testing.assert_array_equal(B[valid], G["rest_B"][valid].astype(np.float32))
    np.testing.assert_array_equal(V, G["rest_V"].astype(np.float32))
    assert (V < 0).any() and (V > 0).any()


def test_oracle_rest_matches_reference():
    """The oracle's precompute_rest (FP64 and FP32) against the reference's
    rest matrices on the non-degenerate tets.  The reference rounds the edge
    differences and B to float32, so even the FP64 oracle differs from it by
    a few float32 ulps."""
    ok = G["rest_valid"].copy()
    ok[-2:] = False
    tets = G["tets"][ok]
    for prec, tol in (("f64", 5e-7), ("f32", 2e-6)):
        rv, B, mass, tot = O.precompute_rest(G["pos0"], tets, 1.0, prec)
        ref = G["rest_B"][ok].astype(np.float64)
        rel = np.abs(B.astype(np.float64) - ref).max() / np.abs(ref).max()
        assert rel <= tol, (prec, rel)


def test_constraint_table_bit_exact():
    """_collect_raw_constraints (builder.py:610-656) -> the reference's SoA
    columns (engine.py:1179-1211), in the reference's order."""
    cfgs = json.loads(str(G["configs"]))
    t = builder.collect_raw_constraints(G["pos0"], G["tets"], cfgs)
    assert t.n == G["c_type"].shape[0]
    for f in ("type", "pts", "stiffness", "compressionstiffness", "dampingratio", "tetid", "L", "restlength",
              "restvector", "restdir"):
        np.testing.assert_array_equal(getattr(t, "c_" + f), G["c_" + f], err_msg=f)


def test_constraint_table_sorted_ranges():
    """musclesim.py:365-396: stable sort by type tag, contiguous per-type ranges."""
    cfgs = json.loads(str(G["configs"]))
    t = builder.collect_raw_constraints(G["pos0"], G["tets"], cfgs).sorted_by_type()
    order = np.argsort(G["c_type"], kind="stable")
    np.testing.assert_array_equal(t.c_pts, G["c_pts"][order])
    np.testing.assert_array_equal(t.c_restlength, G["c_restlength"][order])
    for ty, (off, cnt) in t.cons_ranges.items():
        assert (t.c_type[off:off + cnt] == int(ty)).all() and cnt == (G["c_type"] == int(ty)).sum()


def test_fix_tet_winding_bit_exact():
    np.testing.assert_array_equal(fix_tet_winding(G["pos0"], G["tets"][:-2]), G["tets_fixed"])


@pytest.mark.parametrize("i", range(0, 62, 7))
def test_ramp_activation_bit_exact(i):
    f = int(G["act_frames"][i])
    np.testing.assert_array_equal(ramp_activation(G["act_mask"], f, 1, 50), G["act_values"][i])
