"""Autotuned matvec launch parameters with an on-disk cache.

The library's autotuner (lsg_operator_autotune) times matvecs of one operator
over a candidate set of launch parameters.  Operators of the same dimension,
size class (log2 of the point count and of the cell-operator work, rounded)
and precision share a setting, which this module keeps in a JSON file so
later processes skip the search.
"""
import ctypes
import json
import math
import os

from . import FP32, Tuning, _check, lib


def default_cache():
    return os.environ.get("LSG_TUNING_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "loadsg_b200", "tuning.json"))


def key(matrix, precision):
    info = matrix.info()
    n = max(int(info["n_points"]), 1)
    cells = max(int(info["case_cells"]), 1)
    return f"d{info['d']}-n{round(math.log2(n))}-c{round(math.log2(cells))}-{'fp32' if precision == FP32 else 'fp64'}"


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def autotune(matrix, precision=FP32, reps=3, cache=None):
    path = default_cache() if cache is True else cache
    k = key(matrix, precision)
    if path:
        hit = _load(path).get(k)
        if hit:
            matrix.set_tuning(**hit)
            return hit, None, None
    t = Tuning()
    best = ctypes.c_double(0)
    dflt = ctypes.c_double(0)
    _check(lib().lsg_operator_autotune(matrix._h, precision, reps, ctypes.byref(t), ctypes.byref(best),
                                       ctypes.byref(dflt)))
    setting = t.as_dict()
    if path:
        table = _load(path)
        table[k] = setting
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    return setting, best.value, dflt.value
