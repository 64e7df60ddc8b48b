"""The autotuner's host logic (autotune.py): case-size buckets of the batch,
reading the committed table back, and mapping a tuned shape to the library's
current variant index.  No GPU: the tables are read, not measured."""
import importlib
import json

import pytest


@pytest.fixture(scope="module")
def autotune():
    return importlib.import_module("2d_compressible_flow_solver_b200.autotune")


def test_buckets_by_the_edge_of_a_square_of_the_cells(autotune):
    b = autotune._bucket
    assert b(64, 64) == 96 and b(96, 96) == 96
    assert b(64, 256) == 192          # 128 x 128 cells
    assert b(97, 97) == 192 and b(384, 384) == 384
    assert b(400, 400) == 576 and b(768, 768) == 768
    assert b(1024, 1024) == 768       # past the last edge: the last bucket
    edges = autotune.BATCH_BUCKETS
    assert list(edges) == sorted(edges)


def test_committed_table_gives_rows_for_every_bucket(autotune):
    doc = json.loads(autotune.TABLE.read_text())
    for prec in ("f32", "f64"):
        rows = doc["batch_rows"][prec]["rows"]
        assert set(rows) == {str(e) for e in autotune.BATCH_BUCKETS}
        for nx, ny in [(64, 64), (200, 300), (768, 768)]:
            r = autotune.batch_rows_for(prec, nx, ny)
            assert r == rows[str(autotune._bucket(nx, ny))] and 1 <= r <= 4096


def test_missing_or_malformed_table_means_library_defaults(autotune, tmp_path):
    missing = tmp_path / "none.json"
    assert autotune.batch_rows_for("f32", 64, 64, missing) == 0
    assert autotune.best_variant("f32", 4096 * 4096, missing) == 0
    bad = tmp_path / "bad.json"
    bad.write_text("{not json")
    assert autotune.batch_rows_for("f32", 64, 64, bad) == 0
    assert autotune.best_variant("f32", 4096 * 4096, bad) == 0
    partial = tmp_path / "partial.json"
    partial.write_text(json.dumps({"table": {}}))
    assert autotune.batch_rows_for("f64", 64, 64, partial) == 0
    assert autotune.best_variant("f64", 1024, partial) == 0


def test_best_variant_maps_tuned_shapes_to_current_indices(cfsb, autotune, tmp_path):
    shapes = [tuple(v) for v in cfsb.variants()]
    # a table tuned against a build whose variant numbering differs: index 1
    # there is this build's last shape, index 2 a shape this build lacks
    doc = {"variants": {"1": list(shapes[-1]), "2": [999, 4, 1, 0]},
           "table": {"f32": {"256": {"best": 1}, "4096": {"best": 2}}}}
    path = tmp_path / "t.json"
    path.write_text(json.dumps(doc))
    assert autotune.best_variant("f32", 300 * 300, path) == len(shapes)   # nearest tuned size: 256
    assert autotune.best_variant("f32", 4000 * 4000, path) == 0           # its shape is not in the library
    assert autotune.best_variant("f64", 256 * 256, path) == 0             # no table for the form


def test_committed_table_names_current_variants(cfsb, autotune):
    current = {tuple(v) for v in cfsb.variants()}
    doc = json.loads(autotune.TABLE.read_text())
    for prec, sizes in doc["table"].items():
        for n, row in sizes.items():
            assert tuple(doc["variants"][str(row["best"])]) in current, (prec, n)
            assert autotune.best_variant(prec, int(n) ** 2) >= 1
