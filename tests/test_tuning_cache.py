"""The autotuner's JSON cache without a GPU: the Python writer (merge, atomic replace), the
library's reader (fmm3d_tuning_reload parses the file and counts entries; unreadable
files are ignored) and the cache-path resolution."""
import json
import os

import pytest


@pytest.fixture()
def F():
    import fmmlib3d_b200 as F
    yield F
    F.set_tuning_cache(None)
    F.tuning_reload()


def _entry(**knobs):
    k = {"m2l_kt": 0, "trans_kt": 0, "tc_variant": 0, "overlap": 0, "p2p_ept": 0}
    k.update(knobs)
    return {"knobs": k, "ms": 1.0}


def test_writer_merges_entries(tmp_path, F):
    from fmmlib3d_b200 import autotune as A
    p = str(tmp_path / "c.json")
    A.write_cache(p, "sig a", _entry(m2l_kt=64))
    A.write_cache(p, "sig b", _entry(trans_kt=4))
    A.write_cache(p, "sig a", _entry(m2l_kt=32))
    data = json.load(open(p))
    assert data["format"] == A.CACHE_FORMAT and data["version"] == 1
    assert set(data["entries"]) == {"sig a", "sig b"}
    assert data["entries"]["sig a"]["knobs"]["m2l_kt"] == 32
    assert not [f for f in os.listdir(tmp_path) if ".tmp" in f]


def test_library_reads_cache(tmp_path, F):
    from fmmlib3d_b200 import autotune as A
    p = str(tmp_path / "c.json")
    for i in range(5):
        A.write_cache(p, "laplace sig %d \"quoted\" \\ end" % i, _entry(m2l_kt=16 * (i + 1), overlap=2))
    F.set_tuning_cache(p)
    assert F.tuning_cache_path() == p
    assert F.tuning_reload() == 5
    A.write_cache(p, "another", _entry())
    assert F.tuning_reload() == 6


@pytest.mark.parametrize("text", ["", "{", "[1, 2]", '{"entries": 3}', '{"entries": {"x": {"knobs": [1]}}}',
                                  '{"entries": {"x": {"knobs": {"m2l_kt": "a"}}}} trailing'])
def test_library_ignores_unusable_files(tmp_path, F, text):
    p = tmp_path / "bad.json"
    p.write_text(text)
    F.set_tuning_cache(str(p))
    n = F.tuning_reload()
    # an entry whose knobs are not an object is skipped; a parse error drops the file
    assert n == 0


def test_cache_path_resolution(tmp_path, F, monkeypatch):
    F.set_tuning_cache(None)
    monkeypatch.delenv("FMM3D_TUNING_CACHE", raising=False)
    assert F.tuning_cache_path() == os.path.join(os.path.dirname(F.LIBPATH), "tuning_cache.json")
    F.set_tuning_cache("")
    assert F.tuning_cache_path() == "" and F.tuning_reload() == 0
    F.set_tuning_cache(str(tmp_path / "missing.json"))
    assert F.tuning_reload() == 0


def test_shipped_cache_is_readable(F):
    """The cache shipped beside the library (tuned on a B200) parses and names only known knobs."""
    from fmmlib3d_b200 import TUNING_KNOBS
    from fmmlib3d_b200 import autotune as A
    p = os.path.join(os.path.dirname(F.LIBPATH), "tuning_cache.json")
    if not os.path.exists(p):
        pytest.skip("no shipped tuning cache")
    ents = A.read_cache(p)
    assert ents
    for sig, e in ents.items():
        assert sig.startswith("laplace ") and set(e["knobs"]) == set(TUNING_KNOBS)
    F.set_tuning_cache(p)
    assert F.tuning_reload() == len(ents)


def test_candidates_cover_each_form():
    from fmmlib3d_b200 import autotune as A
    for form in ("fp64-rotation", "fp64-dense", "mixed-cuda", "mixed-tc"):
        names = [k for k, _ in A.candidates(form)]
        assert "trans_kt" in names and "overlap" in names
        assert ("p2p_ept" in names) == form.startswith("mixed")
        assert ("tc_variant" in names) == (form == "mixed-tc")
