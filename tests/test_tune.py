"""The batching autotuner (pgxc/tune.py): workload classes, choice of the
best candidate and the committed table's format."""
import json
import os

from pgxc import cases, tune


def test_buckets_and_keys():
    assert tune.bucket(10, (64, 256)) == 0
    assert tune.bucket(64, (64, 256)) == 0
    assert tune.bucket(65, (64, 256)) == 1
    assert tune.bucket(1000, (64, 256)) == 2
    c = cases.config(2)
    k = tune.single_key(c.nbas, c.npts, "mixed")
    assert k.startswith("single:mixed:nbas") and "npts" in k
    assert tune.set_key(68_000_000) == "set:mixed:npts3"


def test_best_prefers_fastest_then_larger_chunks():
    assert tune.best({65536: 3.0, 262144: 2.0, 0: 2.5}) == 262144
    assert tune.best({65536: 2.0, 262144: 2.0}) == 262144
    assert tune.best({65536: 2.0, 0: 2.0}) == 0          # 0 = as large as memory allows
    assert tune.best({65536: None, 262144: 4.0}) == 262144
    assert tune.best({65536: None}) is None


def test_tune_single_and_choose_round_trip(tmp_path):
    c = cases.config(1)
    fake = {65536: 5.0, 262144: 4.0, 1 << 20: 4.5, 0: 6.0}
    key, t, b = tune.tune_single(c, "mixed", lambda case, prec, chunk: fake[chunk])
    assert b == 262144 and t == fake
    path = str(tmp_path / "t.json")
    tune.write({key: {"max_chunk_points": b, "ms": t[b]}}, path, "test")
    table = tune.load(path)
    assert tune.choose_single(c, "mixed", table) == 262144
    assert tune.choose_single(c, "fp64", table) == 0       # class not in the table: the default


def test_committed_table_is_well_formed():
    if not os.path.exists(tune.TABLE):
        return
    d = json.load(open(tune.TABLE))
    assert set(d) >= {"entries", "candidates", "nbas_edges", "npts_edges"}
    for k, e in d["entries"].items():
        assert k.startswith(("single:", "set:"))
        assert e["max_chunk_points"] in d["candidates"]
