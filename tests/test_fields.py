"""UNSBIN field files: the host library's writer and reader against the reference's compiled
uns::io::write_fields / read_fields (CPU).  Files written by both from the same records are identical
byte for byte, and each side reads the other's files."""
import os

import numpy as np
import pytest

from mpcns_uns_b200 import fields

ref = pytest.importorskip("oracle.ref")
if not ref.available():
    pytest.skip("reference checker not built (make -C oracle ref)", allow_module_level=True)


def _records(rng):
    # odd name lengths and value counts exercise the 8-byte padding; an empty field and a node scalar
    return [fields.FieldRecord("U_H", fields.DIM_CELL, 5, rng.standard_normal(5 * 37)),
            fields.FieldRecord("B", fields.DIM_FACE, 1, rng.standard_normal(81)),
            fields.FieldRecord("J_cell", fields.DIM_CELL, 3, rng.standard_normal(3 * 37)),
            fields.FieldRecord("e", fields.DIM_EDGE, 1, np.zeros(0)),
            fields.FieldRecord("_time", fields.DIM_NODE, 1, np.array([2.5e-3]))]


def test_write_matches_reference_bytes(tmp_path):
    rng = np.random.default_rng(1)
    recs = _records(rng)
    ours, theirs = os.path.join(tmp_path, "ours.unsb"), os.path.join(tmp_path, "ref.unsb")
    fields.write_fields(ours, 0x1234_5678_9ABC_DEF0, recs)
    ref.write_fields(theirs, 0x1234_5678_9ABC_DEF0, [(r.name, r.dim, r.ncomp, r.values) for r in recs])
    assert open(ours, "rb").read() == open(theirs, "rb").read()


def test_each_side_reads_the_other(tmp_path):
    rng = np.random.default_rng(2)
    recs = _records(rng)
    ours, theirs = os.path.join(tmp_path, "ours.unsb"), os.path.join(tmp_path, "ref.unsb")
    fields.write_fields(ours, 77, recs)
    ref.write_fields(theirs, 78, [(r.name, r.dim, r.ncomp, r.values) for r in recs])
    got, h = ref.read_fields(ours)
    assert h == 77 and [g[0] for g in got] == [r.name for r in recs]
    for g, r in zip(got, recs):
        assert (g[1], g[2]) == (r.dim, r.ncomp) and np.array_equal(g[3], r.values)
    back, h = fields.read_fields(theirs)
    assert h == 78 and [b.name for b in back] == [r.name for r in recs]
    for b, r in zip(back, recs):
        assert (b.dim, b.ncomp) == (r.dim, r.ncomp) and np.array_equal(b.values, r.values)


def test_init_fields_and_errors(tmp_path):
    rng = np.random.default_rng(3)
    path = os.path.join(tmp_path, "init.unsb")
    recs = _records(rng)
    recs.append(fields.FieldRecord("U_Na", fields.DIM_CELL, 5, rng.standard_normal(5 * 37)))
    fields.write_fields(path, 0, recs)
    UH, UNa, B, t = fields.read_init_fields(path)
    assert np.array_equal(UH, recs[0].values) and np.array_equal(UNa, recs[-1].values)
    assert np.array_equal(B, recs[1].values) and t == 2.5e-3
    fields.write_fields(path, 0, recs[:2])
    with pytest.raises(RuntimeError, match="lacks U_H, U_Na or B"):
        fields.read_init_fields(path)
    bad = os.path.join(tmp_path, "bad.unsb")
    open(bad, "wb").write(b"NOTUNSBIN" + bytes(32))
    with pytest.raises(RuntimeError, match="not an UNSBIN file"):
        fields.read_fields(bad)
    with pytest.raises(RuntimeError, match="multiple of ncomp"):
        fields.write_fields(path, 0, [fields.FieldRecord("x", fields.DIM_CELL, 3, np.zeros(4))])
