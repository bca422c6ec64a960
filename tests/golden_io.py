"""Loader for the golden fixtures written by tests/golden/make_golden.py."""
import glob
import json
import os

import numpy as np

from conftest import load_package

load_package()
from croma_fp_b200 import config as _config  # noqa: E402

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _names():
    return sorted(os.path.basename(p)[7:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "golden_*.npz")))


def case_names():
    """Snapshot cases (evolve fixtures); the DSA, emission and real-history
    fixtures have their own tests."""
    return [n for n in _names() if not n.startswith(("dsa_", "emission_", "histories"))]


def dsa_case_names():
    """DSA-injection fixtures."""
    return [n for n in _names() if n.startswith("dsa_")]


DSA_COMBOS = [(m, mode, r) for m in (0, 1) for mode in (1, 2) for r in (0, 1, 2)]


class DsaCase:
    """One DSA fixture: inputs and the reference's outputs for every
    (shock form m, injection mode, reacceleration mode) combination."""

    def __init__(self, name):
        self.name = name
        d = np.load(os.path.join(GOLDEN_DIR, f"golden_{name}.npz"))
        self.d = d
        self.nb = int(d["nb"])
        self.ntracer = int(d["ntracer"])
        self.cfg = _config.config1(nb=self.nb)
        self.dt = float(d["dt"])

    def shocks(self, merged):
        pre = f"shock{merged}_"
        out = {k[len(pre):]: self.d[k] for k in self.d.files if k.startswith(pre)}
        out["has_dsa"] = int(out.get("has_dsa", 0))
        return out

    @staticmethod
    def params(reacc):
        return _config.DsaParams(reacc_eta_cap=0.05 if reacc == 2 else 0.0)

    def expected(self, merged, mode, reacc):
        t = f"m{merged}_mode{mode}_r{reacc}"
        d = self.d
        return dict(crp=d[f"{t}_crp"], cre=d[f"{t}_cre"], qpi=d[f"{t}_qpi"], qepri=d[f"{t}_qepri"],
                    dis=d[f"{t}_dis"], ninj=int(d[f"{t}_ninj"]))


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
