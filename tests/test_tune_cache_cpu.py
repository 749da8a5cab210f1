"""Host logic of the persisted autotuner cache (skgemm_tune_cache_save /
_load / _clear), no GPU: a file written by hand loads, saving writes back
the same entries, keys of any length survive, clearing empties the cache,
and malformed files are refused with nothing loaded."""
import json

import pytest

import skgemm


def entry(key, tile=128, order=2, grid=0, ozaki="0"):
    return {"key": key, "tile": tile, "order": order, "grid": grid, "ozaki": ozaki}


def write(path, entries, fmt="skgemm-tune-cache/1"):
    # The library's own layout: a header line, then one entry per line.
    lines = ['{"format": "%s", "entries": [' % fmt]
    for i, e in enumerate(entries):
        lines.append(json.dumps(e) + ("," if i + 1 < len(entries) else ""))
    lines.append("]}")
    path.write_text("\n".join(lines) + "\n")


@pytest.fixture(autouse=True)
def empty_cache():
    skgemm.tune_cache_clear()
    yield
    skgemm.tune_cache_clear()


def test_empty_cache_saves_a_valid_empty_file(tmp_path):
    p = tmp_path / "t.json"
    assert skgemm.tune_cache_save(p) == 0
    doc = json.loads(p.read_text())
    assert doc == {"format": "skgemm-tune-cache/1", "entries": []}


def test_load_save_round_trip(tmp_path):
    long_key = "NVIDIA B200|0,0,0,0,0|" + "".join(f"1:{m}:{m}:110592;" for m in range(16, 4000, 7))
    assert len(long_key) > 4096  # longer than one read buffer
    entries = [entry("NVIDIA B200|0,0,0,0,0|0:512:512:110592;", 64, 1, 0, "0"),
               entry("NVIDIA B200|0,0,0,2,0|1:512:512:110592;0:512:512:110592;", 128, 2, 0,
                     "11"),
               entry(long_key, 128, 2, 296, "0" * 570)]
    src = tmp_path / "in.json"
    write(src, entries)
    assert skgemm.tune_cache_load(src) == 3
    out = tmp_path / "out.json"
    assert skgemm.tune_cache_save(out) == 3
    doc = json.loads(out.read_text())
    assert doc["format"] == "skgemm-tune-cache/1"
    assert sorted(doc["entries"], key=lambda e: e["key"]) == sorted(entries,
                                                                    key=lambda e: e["key"])
    # loading the saved file again is idempotent
    assert skgemm.tune_cache_load(out) == 3
    out2 = tmp_path / "out2.json"
    assert skgemm.tune_cache_save(out2) == 3
    assert out2.read_text() == out.read_text()


def test_clear(tmp_path):
    src = tmp_path / "in.json"
    write(src, [entry("k|0,0,0,0,0|0:64:64:64;")])
    assert skgemm.tune_cache_load(src) == 1
    skgemm.tune_cache_clear()
    out = tmp_path / "out.json"
    assert skgemm.tune_cache_save(out) == 0


@pytest.mark.parametrize("bad", [
    {"fmt": "something-else/1", "entries": [entry("k")]},
    {"entries": [entry("k", tile=96)]},
    {"entries": [entry("k", grid=-1)]},
    {"entries": [entry("k", ozaki="012")]},
    {"entries": [{"key": "k", "tile": 128, "order": 2}]},
    {"entries": [entry("k", order=-3)]},
])
def test_malformed_files_refused_and_nothing_loaded(tmp_path, bad):
    p = tmp_path / "bad.json"
    write(p, [entry("good|0,0,0,0,0|0:64:64:64;")] + bad["entries"],
          bad.get("fmt", "skgemm-tune-cache/1"))
    with pytest.raises(skgemm.SkgemmError) as e:
        skgemm.tune_cache_load(p)
    assert e.value.code == skgemm.ERR_INVALID_ARG
    out = tmp_path / "out.json"
    assert skgemm.tune_cache_save(out) == 0  # the good entry before the bad one too


def test_missing_and_unwritable_paths(tmp_path):
    with pytest.raises(skgemm.SkgemmError):
        skgemm.tune_cache_load(tmp_path / "missing.json")
    with pytest.raises(skgemm.SkgemmError):
        skgemm.tune_cache_save(tmp_path / "no" / "such" / "dir.json")
