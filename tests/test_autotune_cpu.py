"""Host logic of the tile autotuner: its (eps, m) candidates are the
reference's own formula (processing/tomo.py:39-42), its cache round-trips and
batch signatures are stable."""
import numpy as np

from model_mosaic_b200 import autotune
from oracle.usfft import usfft_params


def test_candidates_follow_reference_formula():
    for n in (64, 512, 768, 1024, 1536, 2048, 3072, 24576):
        for eps, m in autotune.CANDIDATES:
            assert usfft_params(n, eps)[1] == m
    assert autotune.REFERENCE == (1e-3, 4) and autotune.REFERENCE in autotune.CANDIDATES


def test_cache_round_trip(tmp_path):
    path = str(tmp_path / "sub" / "at.json")
    assert autotune._load(path) == {}
    data = {"dev|n=64|nz=16|T=90|tol=ref": {"choice": [0.001, 4], "ms": {"eps=0.001,m=4": 1.5}}}
    autotune._save(path, data)
    assert autotune._load(path) == data
    (tmp_path / "bad.json").write_text("{not json")
    assert autotune._load(str(tmp_path / "bad.json")) == {}


def test_batch_signature():
    th = lambda k: np.zeros(k, np.float32)
    a = [dict(n=512, theta=th(360)), dict(n=768, theta=th(400), nz=16)]
    b = [dict(n=512, theta=th(360), nz=16), dict(n=768, theta=th(400))]
    assert autotune.batch_signature(a) == autotune.batch_signature(b)           # nz defaults to 16
    assert autotune.batch_signature(a) != autotune.batch_signature(a[::-1])
    assert autotune.batch_signature(a) != autotune.batch_signature([a[0], dict(n=768, theta=th(401))])


def test_admissible_rule():
    errs = {(1e-2, 3): 4.07e-3, (1e-3, 4): 2.73e-4, (1e-5, 6): 0.0}
    lim, ok = autotune.admissible(errs, None)
    assert lim == errs[(1e-3, 4)] and ok == [(1e-3, 4), (1e-5, 6)]      # default: as accurate as the reference
    lim, ok = autotune.admissible(errs, 1e-2)
    assert ok == [(1e-2, 3), (1e-3, 4), (1e-5, 6)]
    lim, ok = autotune.admissible(errs, 1e-4)
    assert ok == [(1e-5, 6)]
