"""The launch-shape tuning table: host logic (no GPU needed)."""
import json

import pytest


def test_table_first_match_and_defaults():
    from masters_final_b200 import _lib
    L = _lib.load()
    try:
        L.eacb_tune_clear()
        assert L.eacb_tune_get(0, 16, 500_000, 2) == 2            # no entry: the default
        assert L.eacb_tune_set(0, 16, 16, 250_000, 1_000_000, 1) == 0
        assert L.eacb_tune_set(0, 1, 32, 0, 10 ** 12, 2) == 0
        assert L.eacb_tune_get(0, 16, 500_000, 7) == 1            # the first matching entry
        assert L.eacb_tune_get(0, 8, 500_000, 7) == 2
        assert L.eacb_tune_get(1, 16, 500_000, 7) == 7            # another knob
        assert _lib.status_string(L.eacb_tune_set(99, 0, 0, 0, 0, 1)) == "EACB_ERR_BAD_ARGUMENT"
        assert _lib.status_string(L.eacb_tune_set(0, 5, 4, 0, 0, 1)) == "EACB_ERR_BAD_ARGUMENT"
    finally:
        _lib.apply_tuning()


def test_apply_tuning_file(tmp_path):
    from masters_final_b200 import _lib
    L = _lib.load()
    p = tmp_path / "t.json"
    p.write_text(json.dumps({"entries": [{"knob": "mst_phase1_permille", "a": [0, 0],
                                          "b": [1, 10 ** 9], "value": 125}],
                             "python": {"batched_workers": 24}}))
    try:
        assert _lib.apply_tuning(str(p)) == 1
        assert L.eacb_tune_get(_lib.TUNE_KNOBS["mst_phase1_permille"], 0, 1000, 250) == 125
        assert _lib.tuned("batched_workers", 16) == 24
        _lib.clear_tuning()
        assert L.eacb_tune_get(_lib.TUNE_KNOBS["mst_phase1_permille"], 0, 1000, 250) == 250
        assert _lib.tuned("batched_workers", 16) == 16
        p.write_text(json.dumps({"entries": [{"knob": "no_such_knob", "a": [0, 0],
                                              "b": [0, 0], "value": 1}]}))
        with pytest.raises(KeyError):
            _lib.apply_tuning(str(p))
    finally:
        _lib.apply_tuning()


def test_committed_table_loads():
    """The table the autotuner wrote for this package is well formed: known
    knobs, ordered ranges, values in each knob's range."""
    import os
    from masters_final_b200 import _lib
    if not os.path.exists(_lib.TUNING_PATH):
        pytest.skip("no tuning table in this checkout")
    with open(_lib.TUNING_PATH) as f:
        table = json.load(f)
    allowed = {"tc_ctas_per_sm": {1, 2, 4}, "tc_buffers": {1, 2}, "co_count_ctas": {1, 2},
               "co_fill_ctas": {1, 2}, "co_dense_ratio": {4, 16, 64}}
    for e in table["entries"]:
        assert e["knob"] in _lib.TUNE_KNOBS
        assert e["a"][0] <= e["a"][1] and e["b"][0] <= e["b"][1]
        if e["knob"] in allowed:
            assert e["value"] in allowed[e["knob"]]
        assert e["timings"]
    assert _lib.apply_tuning() == len(table["entries"])
