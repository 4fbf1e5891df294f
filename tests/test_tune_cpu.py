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
