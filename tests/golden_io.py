"""Loader for the golden fixtures written by tests/golden/make_golden.py."""
import glob
import json
import os

import numpy as np

from conftest import load_package

load_package()
from croma_fp_b200 import config as _config  # noqa: E402

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def case_names():
    return sorted(os.path.basename(p)[7:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "golden_*.npz")))


class Case:
    def __init__(self, name):
        self.name = name
        d = np.load(os.path.join(GOLDEN_DIR, f"golden_{name}.npz"))
        self.d = d
        self.cfg = _config.RunConfig(**json.loads(str(d["config"])))
        self.ntracer = int(d["ntracer"])
        self.isnap0 = int(d["isnap0"])
        self.nrun = int(d["nrun"])
        self.nsnap = int(d["nsnap"])

    def snapshot_args(self, k):
        """(bg_curr, bg_next, z_curr, z_next, allow, dt, elapsed) of run step k."""
        d = self.d
        isnap = self.isnap0 + k
        allow = isnap + 1 < self.nsnap
        cur = d["bg"][k]
        nxt = d["bg"][k + 1] if allow else cur
        z_next = float(d["z"][isnap + 1]) if allow else float(d["z"][isnap])
        return cur, nxt, float(d["z"][isnap]), z_next, allow, float(d["dt"][isnap]), float(d["elapsed"][isnap])


def rel_err(x, y, floor_frac=1e-12):
    """Max relative error of x vs y on bins above floor_frac x per-row peak
    of |y| (rows are tracers)."""
    x = np.asarray(x, dtype=np.float64); y = np.asarray(y, dtype=np.float64)
    peak = np.max(np.abs(y), axis=-1, keepdims=True)
    mask = np.abs(y) > floor_frac * peak
    if not mask.any():
        return float(np.max(np.abs(x - y)))
    return float(np.max(np.abs(x - y)[mask] / np.abs(y)[mask]))
