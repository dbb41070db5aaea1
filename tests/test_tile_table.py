"""The batched-GEMM tile table (hm_tile_table_load): the JSON autotune.py writes is
accepted, anything else is refused with HM_ERR_ARG and leaves the table as it was.
Host-only: no GPU needed."""
import json
import os

import pytest

import hmat_b200 as H


@pytest.fixture
def lib():
    L = H.load()
    yield L
    L.hm_tile_table_load(b"")


def test_valid_table_loads(tmp_path, lib):
    t = {"factor.update_correct|f32|p1024|m256|n96|k128": [64, 1, 0],
         "solve.project|f64|p512|m512|n64|k256": [128, 0, 1]}
    f = tmp_path / "t.json"
    f.write_text(json.dumps(t, indent=1))
    assert lib.hm_tile_table_load(str(f).encode()) == H.HM_OK
    assert lib.hm_tile_table_size() == 2
    f.write_text("{}")
    assert lib.hm_tile_table_load(str(f).encode()) == H.HM_OK
    assert lib.hm_tile_table_size() == 0


@pytest.mark.parametrize("text", [
    '{"a": [48, 0, 0]}',          # bn not a tile width
    '{"a": [64, 4, 0]}',          # shape not 0-3
    '{"a": [64, 0]}',             # too short
    '{"a": [64, 0, 0] "b": [32, 0, 0]}',
    '["a", 64, 0, 0]',
    '',
])
def test_malformed_tables_are_refused(tmp_path, lib, text):
    good = tmp_path / "good.json"
    good.write_text('{"x|f32|p1|m1|n32|k1": [32, 0, 0]}')
    assert lib.hm_tile_table_load(str(good).encode()) == H.HM_OK
    bad = tmp_path / "bad.json"
    bad.write_text(text)
    assert lib.hm_tile_table_load(str(bad).encode()) == H.HM_ERR_ARG
    assert lib.hm_tile_table_size() == 1      # unchanged


def test_missing_file_and_clear(tmp_path, lib):
    assert lib.hm_tile_table_load(str(tmp_path / "none.json").encode()) == H.HM_ERR_ARG
    assert lib.hm_tile_table_load(b"") == H.HM_OK
    assert lib.hm_tile_table_size() == 0
    with pytest.raises(H.HmError):
        H.tile_table_load(str(tmp_path / "none.json"))


def test_committed_table_is_valid(lib):
    path = os.path.join(os.path.dirname(H.__file__), "tile_table.json")
    with open(path) as f:
        entries = json.load(f)
    assert lib.hm_tile_table_load(path.encode()) == H.HM_OK
    assert lib.hm_tile_table_size() == len(entries) > 0
