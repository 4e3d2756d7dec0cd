"""Host logic of the autotuner that needs no GPU: candidate generation, the
cache key, the cache file round trip and reading older cache entries."""

import json

from lowrank_gpu_fastest_b200 import tune


def test_candidates_respect_thread_and_brick_limits():
    for T, stride in ((48, 3), (96, 2), (128, 1)):
        c = tune.candidates(T, (11, 11, 11), stride)
        assert c, "no candidates"
        assert len(c) == len(set(c)), "duplicate candidates"
        for (bx, by, bz), split in c:
            assert 27 <= bx * by * bz * split <= 256
            assert bx <= 8 and by <= 8
            assert split in ((2, 4) if T <= 96 else (4,))
        # the stride lattice is among the brick sides
        assert any(b[0] == stride and b[1] == stride for b, _ in c)


def test_cache_key_names_every_dimension():
    k = tune.key("sm_100:148", 48, (11, 11, 11), 3, "plain")
    assert k == "v2|sm_100:148|T48|p11x11x11|s3|plain"
    assert tune.key("sm_100:148", 48, (11, 11, 11), 3, "tensor") != k
    assert tune.key("sm_100:148", 48, (7, 7, 7), 3, "plain") != k
    assert tune.key("sm_100:148", 64, (11, 11, 11), 3, "plain") != k
    assert tune.key("sm_100:148", 48, (11, 11, 11), 2, "plain") != k


def test_cache_file_round_trip_and_older_entries(tmp_path, monkeypatch):
    path = tmp_path / "sub" / "tune.json"
    monkeypatch.setenv("LRD_TUNE_CACHE", str(path))
    assert tune.cache_path() == str(path)
    assert tune._load() == {}
    entry = {"brick": [3, 3, 3], "split": 2, "gram_split": 4, "eigh_block": 1, "recon_ms": 1.0}
    tune._save({"k": entry})
    assert json.load(open(path)) == {"k": entry}
    assert tune._load() == {"k": entry}
    assert tune._choice(entry) == dict(brick=(3, 3, 3), split=2, gram_split=4, eigh_block=1)
    # an entry written before the Gram split and the eigensolver schedule were
    # tuned reads as the plan's own choices for those
    assert tune._choice({"brick": [2, 2, 8], "split": 4}) == dict(brick=(2, 2, 8), split=4, gram_split=0,
                                                                  eigh_block=0)
    # a damaged cache file reads as empty
    path.write_text("{not json")
    assert tune._load() == {}
