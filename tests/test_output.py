"""Output files and checkpoints (include/croma_b200_output.h) against the
reference's own writers (src/tracer_fp_output.c, src/tracer_fp_restart.c,
compiled into oracle/_ref): the files must be identical byte for byte.

CPU: tile and mapped layouts, CR state (electrons and protons) and emission
rows, with and without the per-cm^3 volume factor, reopened with
resume_existing; the TFPCHK1 checkpoint writer and reader, including the
metadata and tracer-order checks.  GPU: slabs written straight from a
context's resident spectra (asynchronous staging, copy stream, writer
thread) equal the host writer's files, and a checkpoint of the device state
restores it.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

from conftest import load_package

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "oracle"))
import pyoracle  # noqa: E402

load_package()
from croma_fp_b200 import config, output  # noqa: E402

NB = 128


def _ref():
    if not pyoracle.reference_available(NB):
        pytest.skip("oracle/_ref not built")
    return pyoracle.ReferenceCPU(config.config1(nb=NB))


def _p(a):
    return None if a is None else a.ctypes.data


def _data(n, seed):
    rng = np.random.default_rng(seed)
    cre = rng.lognormal(0.0, 3.0, (n, NB)) * 1e-20
    crp = rng.lognormal(0.0, 3.0, (n, NB)) * 1e-22
    rho = rng.uniform(1e-30, 1e-26, n)
    rho[3] = 0.0
    rho[5] = -1.0
    mass = rng.uniform(1e6, 1e8, n)
    mass[7] = 0.0
    return cre, crp, rho, mass


def _bytes(path):
    with open(path, "rb") as f:
        return f.read()


@pytest.mark.parametrize("per_cc", [0, 1])
def test_tile_files_match_reference(tmp_path, per_cc):
    L = _ref().lib
    n, nsnap, nfreq = 11, 3, 5
    ours, refd = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    refd.mkdir()
    cre_out = output.OutputFile(NB, str(ours), "CRE", 2, "tile", nsnap + 1, n, NB)
    crp_out = output.OutputFile(NB, str(ours), "CRP", 2, "tile", nsnap + 1, n, NB)
    syn_out = output.OutputFile(NB, str(ours), "eSyn", 2, "tile", nsnap, n, nfreq)
    he = L.ref_tile_open(str(refd).encode(), b"CRE", 2, nsnap + 1, n, NB, 0)
    hp = L.ref_tile_open(str(refd).encode(), b"CRP", 2, nsnap + 1, n, NB, 0)
    hs = L.ref_tile_open(str(refd).encode(), b"eSyn", 2, nsnap, n, nfreq, 0)
    assert min(he, hp, hs) >= 0
    for slab in (0, 2, 3):
        cre, crp, rho, mass = _data(n, slab)
        cre_out.write(slab, cre, rho, mass, per_cc)
        crp_out.write(slab, crp, rho, mass, per_cc)
        assert L.ref_tile_write_cr(he, hp, n, slab, _p(cre), _p(crp), _p(rho), _p(mass), per_cc, 1) == 0
        if slab < nsnap:
            eps = np.ascontiguousarray(cre[:, :nfreq] * 1e3)
            syn_out.write(slab, eps, rho, mass, per_cc)
            assert L.ref_tile_write_emit(hs, n, slab, nfreq, _p(eps), _p(rho), _p(mass), per_cc) == 0
    for o in (cre_out, crp_out, syn_out):
        o.close()
    for h in (he, hp, hs):
        assert L.ref_tile_close(h) == 0
    for stem in ("CRE", "CRP", "eSyn"):
        a, b = _bytes(ours / f"{stem}_tile_core02.bin"), _bytes(refd / f"{stem}_tile_core02.bin")
        assert len(a) == len(b) and a == b, stem
    # reopened with resume_existing: one more slab, still identical
    cre, crp, rho, mass = _data(n, 9)
    with output.OutputFile(NB, str(ours), "CRE", 2, "tile", nsnap + 1, n, NB, resume_existing=True) as o:
        o.write(1, cre, rho, mass, per_cc)
    h = L.ref_tile_open(str(refd).encode(), b"CRE", 2, nsnap + 1, n, NB, 1)
    assert L.ref_tile_write_cr(h, -1, n, 1, _p(cre), None, _p(rho), _p(mass), per_cc, 0) == 0
    assert L.ref_tile_close(h) == 0
    assert _bytes(ours / "CRE_tile_core02.bin") == _bytes(refd / "CRE_tile_core02.bin")
    # a file of another size is refused on resume
    with pytest.raises(output.OutputError):
        output.OutputFile(NB, str(ours), "CRE", 2, "tile", nsnap + 2, n, NB, resume_existing=True)


@pytest.mark.parametrize("per_cc", [0, 1])
def test_mapped_files_match_reference(tmp_path, per_cc):
    L = _ref().lib
    n, nsnap, nbin = 9, 4, 6
    ours, refd = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    refd.mkdir()
    cre_out = output.OutputFile(NB, str(ours), "CRE", 0, "mapped", nsnap + 1, n, NB)
    crp_out = output.OutputFile(NB, str(ours), "CRP", 0, "mapped", nsnap + 1, n, NB)
    ic_out = output.OutputFile(NB, str(ours), "eIC", 0, "mapped", nsnap, n, nbin)
    he = L.ref_map_open(str(refd).encode(), b"CRE", 0, n, (nsnap + 1) * NB, 0)
    hp = L.ref_map_open(str(refd).encode(), b"CRP", 0, n, (nsnap + 1) * NB, 0)
    hi = L.ref_map_open(str(refd).encode(), b"eIC", 0, n, nsnap * nbin, 0)
    assert min(he, hp, hi) >= 0
    for slot in (0, 1, 4):
        cre, crp, rho, mass = _data(n, 10 + slot)
        cre_out.write(slot, cre, rho, mass, per_cc)
        crp_out.write(slot, crp, rho, mass, per_cc)
        assert L.ref_write_cr_map(he, hp, n, slot, _p(cre), _p(crp), _p(rho), _p(mass), per_cc) == 0
        if slot < nsnap:
            eps = np.ascontiguousarray(crp[:, 10:10 + nbin])
            ic_out.write(slot, eps, rho, mass, per_cc)
            assert L.ref_write_emit_map(hi, n, slot, nbin, _p(eps), _p(rho), _p(mass), per_cc) == 0
    for o in (cre_out, crp_out, ic_out):
        o.close()
    for h in (he, hp, hi):
        assert L.ref_map_close(h) == 0
    for stem in ("CRE", "CRP", "eIC"):
        a, b = _bytes(ours / f"{stem}_core00.bin"), _bytes(refd / f"{stem}_core00.bin")
        assert len(a) == len(b) and a == b, stem


def test_checkpoint_matches_reference_and_checks_metadata(tmp_path):
    L = _ref().lib
    n = 13
    cre, crp, _, _ = _data(n, 21)
    ids = np.arange(1000, 1000 + n, dtype=np.int32)[::-1].copy()
    meta = dict(rank=1, world=4, ntracer_global=52, nsnap=40, nfreq=64, nsnp_i=3, nsnp_f=43, tracer_start=13)
    ours, refd = tmp_path / "ours", tmp_path / "ref"
    output.checkpoint_write_host(NB, str(ours), crp, cre, ids, completed=17, **meta)
    assert L.ref_ckpt_write(str(refd).encode(), 1, 4, n, 52, 40, 64, 17, 13, _p(ids), _p(crp), _p(cre),
                            3, 43) == 0
    a, b = _bytes(ours / "checkpoint_rank01.bin"), _bytes(refd / "checkpoint_rank01.bin")
    assert a == b and len(a) == 72 + 4 * n + 2 * 8 * n * NB
    assert not (ours / "checkpoint_rank01.bin.tmp").exists()
    # ours reads the reference's file and the reference reads ours
    r_crp, r_cre, done = output.checkpoint_read_host(NB, str(refd), ids, **meta)
    assert done == 17 and np.array_equal(r_crp, crp) and np.array_equal(r_cre, cre)
    x_crp, x_cre, x_done = np.empty_like(crp), np.empty_like(cre), C.c_int()
    assert L.ref_ckpt_read(str(ours).encode(), 1, 4, n, 52, 40, 64, 13, _p(ids), _p(x_crp), _p(x_cre), 3, 43,
                           C.byref(x_done)) == 0
    assert x_done.value == 17 and np.array_equal(x_crp, crp)
    # metadata and order mismatches are refused
    with pytest.raises(output.OutputError, match="metadata"):
        output.checkpoint_read_host(NB, str(ours), ids, **dict(meta, nfreq=32))
    with pytest.raises(output.OutputError, match="metadata"):
        output.checkpoint_read_host(NB, str(ours), ids, **dict(meta, nsnap=17))
    with pytest.raises(output.OutputError, match="order"):
        output.checkpoint_read_host(NB, str(ours), ids[::-1].copy(), **meta)


@pytest.mark.gpu
def test_device_state_outputs_and_checkpoint(tmp_path):
    from croma_fp_b200 import native, synth
    cfg = config.config1(nb=NB)
    n, nsnap = 300, 3
    w = synth.Workload(cfg, n, 100, seed=31)
    fp = native.TracerFP(cfg, path="fused")
    try:
        gp, ge = fp.grid(0), fp.grid(1)
        crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), n, cfg.species)
        fp.set_state(crp, cre, mass=w.mass)
        dev, host = tmp_path / "dev", tmp_path / "host"
        dev.mkdir()
        host.mkdir()
        files = {}
        for d in (dev, host):
            files[d] = (output.OutputFile(NB, str(d), "CRE", 0, "tile", nsnap + 1, n, NB),
                        output.OutputFile(NB, str(d), "CRP", 0, "mapped", nsnap + 1, n, NB))
        rng = np.random.default_rng(3)
        for k in range(nsnap + 1):
            rho = rng.uniform(1e-29, 1e-27, n)
            per_cc = k % 2
            if k > 0:
                fp.snapshot(*w.snapshot_args(20 + k), sync=False)
            # queued from the device state at this point of the stream
            output.OutputFile.write_state(fp, files[dev][0], files[dev][1], k, rho, per_cc)
            s_crp, s_cre = fp.get_state()
            files[host][0].write(k, s_cre, rho, w.mass, per_cc)
            files[host][1].write(k, s_crp, rho, w.mass, per_cc)
        for d in (dev, host):
            for o in files[d]:
                o.close()
        assert _bytes(dev / "CRE_tile_core00.bin") == _bytes(host / "CRE_tile_core00.bin")
        assert _bytes(dev / "CRP_core00.bin") == _bytes(host / "CRP_core00.bin")
        # checkpoint of the device state, then restore into a fresh context
        ids = np.arange(n, dtype=np.int32)
        output.checkpoint_write(fp, str(tmp_path / "ck"), ids, nsnap=nsnap, completed=nsnap - 1)
        g_crp, g_cre = fp.get_state()
    finally:
        fp.close()
    fp2 = native.TracerFP(cfg, path="fused")
    try:
        fp2.set_state(np.zeros((n, NB)), np.zeros((n, NB)), mass=w.mass)
        done = output.checkpoint_read(fp2, str(tmp_path / "ck"), ids, nsnap=nsnap)
        r_crp, r_cre = fp2.get_state()
        assert done == nsnap - 1 and np.array_equal(r_crp, g_crp) and np.array_equal(r_cre, g_cre)
    finally:
        fp2.close()
