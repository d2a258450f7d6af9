"""Launch parameters and the autotuner (lsg_operator_*_tuning, lsg_operator_autotune):
every admissible setting computes the same product (checked against the
reference's golden vectors, FP64 1e-12), the autotuner keeps a valid setting
that is not slower than the one it started from, and its cache round-trips."""
import json

import numpy as np
import pytest

import loadsg_b200 as lsg
from conftest import GOLDEN, load_golden

pytestmark = pytest.mark.gpu

SETTINGS = [
    dict(cell_threads=128),
    dict(cell_space_kb=16),                    # small work space: more slabs chunked
    dict(cell_space_kb=48, class_ratio=2),
    dict(cell_space_kb=200, class_ratio=1024),
    dict(level_threads=32, level_cap=256),     # most wavefront items spill to global scratch
    dict(level_threads=64, level_cap=65536),
    dict(level_threads=512),
    dict(prolong_threads=32),
    dict(prolong_threads=1024, cell_threads=64),
]


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def cases():
    return [load_golden(p) for p in GOLDEN]


def make(c):
    g = lsg.AdaptiveSparseGrid(c["points"], c["active"])
    p = lsg.MidpointDiffusion(int(c["coef_family"]), c["coef_params"])
    return g, p, lsg.MatrixVectorHomogen(g, p)


@pytest.mark.parametrize("setting", SETTINGS, ids=lambda s: ",".join(f"{k}={v}" for k, v in s.items()))
def test_every_setting_matches_reference(cases, setting):
    for c in cases:
        g, p, m = make(c)
        m.set_tuning(**setting)
        assert all(m.tuning()[k] == v for k, v in setting.items())
        y = np.zeros(g.n)
        m.multiplication(c["x"], y, p)
        assert rel(y, c["matvec_y"]) < 1e-12, c["name"]


def test_invalid_settings_are_rejected(cases):
    _, _, m = make(cases[0])
    for bad in (dict(cell_threads=512), dict(cell_threads=100), dict(cell_space_kb=8), dict(class_ratio=1),
                dict(level_threads=1024), dict(level_cap=16), dict(prolong_threads=2048)):
        with pytest.raises(lsg.LsgError):
            m.set_tuning(**bad)


def test_autotune_keeps_a_valid_faster_setting(cases, tmp_path):
    c = next(c for c in cases if c["name"] == "d6_L3")
    g, p, m = make(c)
    cache = str(tmp_path / "tuning.json")
    setting, best, dflt = m.autotune(lsg.FP32, reps=3, cache=cache)
    assert best is not None and best <= dflt * 1.05
    assert m.tuning() == setting
    y = np.zeros(g.n)
    m.multiplication(c["x"], y, p)
    assert rel(y, c["matvec_y"]) < 1e-12
    table = json.load(open(cache))
    assert list(table.values()) == [setting]
    # a second operator of the same class takes the cached setting without a search
    _, _, m2 = make(c)
    setting2, best2, _ = m2.autotune(lsg.FP32, cache=cache)
    assert best2 is None and setting2 == setting and m2.tuning() == setting
