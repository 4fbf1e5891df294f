"""Autotuner bookkeeping without a GPU: configuration listing from the
library, and the persisted database (keys, round trip, lookup by size
bucket)."""
import json

from massively_b200 import tune


def test_every_family_lists_its_configurations():
    for fam in tune.FAMILIES:
        names = tune.configs(fam)
        assert len(names) >= 1 and all(isinstance(n, str) and n for n in names)


def test_database_round_trip_and_buckets(tmp_path):
    path = str(tmp_path / "db.json")
    assert tune.load_db(path) == {}
    key = tune._key("NVIDIA B200", "radix", "u32", 3 << 27)
    assert key == "NVIDIA B200|radix|u32|2^28"
    tune.save_db({key: {"config": 2, "ms": 1.0}}, path)
    assert json.load(open(path))[key]["config"] == 2
    # every size in the same power-of-two bucket finds the record
    assert tune.lookup("NVIDIA B200", "radix", "u32", 1 << 28, path) == 2
    assert tune.lookup("NVIDIA B200", "radix", "u32", (1 << 29) - 1, path) == 2
    assert tune.lookup("NVIDIA B200", "radix", "u32", 1 << 29, path) is None
    assert tune.lookup("NVIDIA B200", "scan", "u32", 1 << 28, path) is None


def test_corrupt_database_reads_as_empty(tmp_path):
    p = tmp_path / "db.json"
    p.write_text("{not json")
    assert tune.load_db(str(p)) == {}


def test_database_lives_outside_the_package(monkeypatch, tmp_path):
    import os

    import massively_b200
    monkeypatch.delenv("MB_TUNE_DB", raising=False)
    monkeypatch.setenv("XDG_CACHE_HOME", str(tmp_path))
    p = tune.default_db_path()
    assert p == os.path.join(str(tmp_path), "massively_b200", "tune_db.json")
    pkg = os.path.dirname(os.path.abspath(massively_b200.__file__))
    assert not os.path.abspath(p).startswith(pkg)
    monkeypatch.setenv("MB_TUNE_DB", str(tmp_path / "x.json"))
    assert tune.default_db_path() == str(tmp_path / "x.json")
    tune.save_db({"k": {"config": 1}})  # creates the folder on demand
    assert tune.load_db() == {"k": {"config": 1}}


def test_segment_length_class_keys_records():
    import numpy as np
    even = tune.segment_class(np.full(1000, 64))
    skew = tune.segment_class(np.random.default_rng(0).lognormal(3.0, 1.5, 1000))
    assert even == "seg:mean2^6:cv0"
    assert even != skew and skew.startswith("seg:")
    assert tune.segment_class([]) == ""
    assert tune._key("D", "seg", "f32", 1 << 26, even) == "D|seg|f32|2^26|seg:mean2^6:cv0"
    assert tune._key("D", "radix", "u32", 1 << 26) == "D|radix|u32|2^26"


def test_shipped_table_backs_the_database(tmp_path):
    # A key the caller's database lacks falls back to the table shipped with
    # the package (device "*"); the caller's own record wins over it.
    path = str(tmp_path / "db.json")
    assert tune.lookup("NVIDIA B200", "radix", "u32/f32", 1 << 27, path) is None
    assert tune.lookup("NVIDIA B200", "radix", "u32/f32", 1 << 27, path, shipped=True) == 9
    key = tune._key("NVIDIA B200", "radix", "u32/f32", 1 << 27)
    tune.save_db({key: {"config": 2, "ms": 1.0}}, path)
    assert tune.lookup("NVIDIA B200", "radix", "u32/f32", 1 << 27, path, shipped=True) == 2
    shipped = json.load(open(tune.SHIPPED_TABLE))
    for k, rec in shipped.items():
        fam = k.split("|")[1]
        assert 0 <= rec["config"] < len(tune.configs(fam))
