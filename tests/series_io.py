"""A tracer snapshot series written from the committed real-history fixture
(tests/golden/golden_histories.npz: the raw fields of 64 tracer_10k tracers
over the series' first 20 snapshots), in the layout of the reference's
snapshot files (one file per snapshot, subset__tracer_z_dumpNNNN.h5, the
fields at the root; src/tracer_fp_background.c:70-146, :955-957,
:1003-1204), so that the series loader, the HDF5 reader and the device
background run on real data where the reference tree is absent."""
from __future__ import annotations

import math
import os

import numpy as np

import h5write
from golden_io import GOLDEN_DIR

FIX = np.load(os.path.join(GOLDEN_DIR, "golden_histories.npz"))
RAW_FIELDS = ("temperature", "density", "B_x", "B_y", "B_z", "div_v", "curl_v", "dx_phys")
NLONG = 20
FIRST = 25   # the series' first file index (dump0025)


def write_series(directory: str, nsnap: int = NLONG) -> list[str]:
    """Files dump0025 .. dump(0025 + nsnap - 1) under directory."""
    paths = []
    mass = FIX["long_mass"]
    for k in range(nsnap):
        c_dens = float(FIX["c_dens"][k])
        tree = {f: np.ascontiguousarray(FIX[f"long{k}_{f}"]) for f in RAW_FIELDS}
        tree["Redshift"] = np.array(float(FIX["z"][k]))
        tree["dUnit"] = np.array(c_dens)
        tree["vUnit"] = np.array(float(FIX["c_mag"][k]) / math.sqrt(4.0 * math.pi * c_dens))
        tree["M_tracer"] = np.ascontiguousarray(mass)
        tree["particle_ID"] = np.arange(100, 100 + mass.shape[0], dtype=np.int64)
        p = os.path.join(directory, f"subset__tracer_z_dump{FIRST + k:04d}.h5")
        h5write.write(p, tree, compact={"Redshift", "dUnit", "vUnit"})
        paths.append(p)
    return paths
