"""solve_cc_cuda_batch_noalloc: the allocation-free batched Chang-Cooper step.

It exists for callers that cannot allocate device memory when they solve
(their device memory already belongs to their own pool allocator, or the
step cannot afford cudaMalloc/cudaFree synchronising the device).  Those
callers own every buffer; the library keeps its only scratch in a fixed
device array.  This test, as such a caller, allocates its device buffers up
front with torch, calls the entry point through the C ABI twice in a row
(with different sizes, so the second call runs over what the first left in
the shared scratch) and checks each result against the allocating entry
point solve_cc_cuda_batch on the same systems.  The file runs last so that
a failure here comes after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import load_package

load_package()
from croma_fp_b200 import native, ref_abi  # noqa: E402

pytestmark = pytest.mark.gpu

_vp, _i, _d = C.c_void_p, C.c_int, C.c_double
MAX_ROWS = 1 << 19


def _lib():
    lib = native.load_library(128)
    lib.solve_cc_cuda_batch_noalloc.argtypes = [_i, _i, _d, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
    lib.croma_b200_last_error.restype = C.c_char_p
    return lib


def _systems(nsys, nrow, seed):
    """Chang-Cooper-like rows: positive couplings, dominant diagonal."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.0, 3.0, (nsys, nrow))
    c = rng.uniform(0.0, 3.0, (nsys, nrow))
    a[:, 0] = 0.0
    c[:, -1] = 0.0
    b = 1.0 + a + c + rng.uniform(0.0, 1.0, (nsys, nrow))
    src = rng.uniform(0.0, 1e3, (nsys, nrow))
    x0 = rng.uniform(1e-3, 1e6, (nsys, nrow))
    return a, b, c, src, x0


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    lib = _lib()
    abi = ref_abi.RefAbi(128)
    stream = torch.cuda.current_stream()
    for nsys, nrow, seed in ((300, 128, 11), (1500, 256, 12)):
        a, b, c, src, x0 = _systems(nsys, nrow, seed)
        dt = 2.5e-3
        inp = ref_abi.FpChangCooperSolveBatchInput(nsys, nrow, dt, ref_abi.dptr(a), ref_abi.dptr(b),
                                                   ref_abi.dptr(c), ref_abi.dptr(src))
        ref = np.empty_like(x0)
        assert abi.lib.solve_cc_cuda_batch(C.byref(inp), ref_abi.dptr(x0), ref_abi.dptr(ref), None, None) == 0
        dev = [torch.from_numpy(v).cuda() for v in (a, b, c, src, x0)]
        out = torch.empty_like(dev[4])
        torch.cuda.synchronize()
        rc = lib.solve_cc_cuda_batch_noalloc(nsys, nrow, dt, *[t.data_ptr() for t in dev], out.data_ptr(),
                                             stream.cuda_stream)
        assert rc == 0, lib.croma_b200_last_error().decode()
        got = out.cpu().numpy()
        rel = np.max(np.abs(got - ref) / np.abs(ref))
        assert rel <= 1e-12, f"no-alloc result differs from solve_cc_cuda_batch: {rel:.3e}"


def test_noalloc_rejects_batches_beyond_its_scratch():
    lib = _lib()
    nrow = 512
    nsys = MAX_ROWS // nrow + 1
    # pointers are never dereferenced: the size check comes first
    rc = lib.solve_cc_cuda_batch_noalloc(nsys, nrow, 1.0, 8, 8, 8, 8, 8, 8, None)
    assert rc == -1
    assert b"524288" in lib.croma_b200_last_error()


def test_noalloc_singular_pivot_then_clean_call():
    """A zero first diagonal in one system gives -2 (the error word at the
    head of the shared scratch is set); the next, valid call clears it and
    returns 0 with the same result as solve_cc_cuda_batch."""
    import torch
    lib = _lib()
    abi = ref_abi.RefAbi(128)
    stream = torch.cuda.current_stream()
    nsys, nrow, dt = 64, 128, 1e-3
    a, b, c, src, x0 = _systems(nsys, nrow, 21)
    bad = b.copy()
    bad[17, 0] = 0.0
    dev = [torch.from_numpy(v).cuda() for v in (a, bad, c, src, x0)]
    out = torch.empty_like(dev[4])
    torch.cuda.synchronize()
    rc = lib.solve_cc_cuda_batch_noalloc(nsys, nrow, dt, *[t.data_ptr() for t in dev], out.data_ptr(),
                                         stream.cuda_stream)
    assert rc == -2
    assert b"singular" in lib.croma_b200_last_error()
    dev[1] = torch.from_numpy(b).cuda()
    torch.cuda.synchronize()
    rc = lib.solve_cc_cuda_batch_noalloc(nsys, nrow, dt, *[t.data_ptr() for t in dev], out.data_ptr(),
                                         stream.cuda_stream)
    assert rc == 0, lib.croma_b200_last_error().decode()
    inp = ref_abi.FpChangCooperSolveBatchInput(nsys, nrow, dt, ref_abi.dptr(a), ref_abi.dptr(b), ref_abi.dptr(c),
                                               ref_abi.dptr(src))
    ref = np.empty_like(x0)
    assert abi.lib.solve_cc_cuda_batch(C.byref(inp), ref_abi.dptr(x0), ref_abi.dptr(ref), None, None) == 0
    got = out.cpu().numpy()
    assert np.max(np.abs(got - ref) / np.abs(ref)) <= 1e-12


def test_noalloc_refuses_a_capturing_stream():
    import torch
    lib = _lib()
    nsys, nrow = 8, 128
    a, b, c, src, x0 = _systems(nsys, nrow, 22)
    dev = [torch.from_numpy(v).cuda() for v in (a, b, c, src, x0)]
    out = torch.empty_like(dev[4])
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    rc = None
    with torch.cuda.graph(g, stream=s):
        out.add_(0.0)   # the captured graph is not empty
        rc = lib.solve_cc_cuda_batch_noalloc(nsys, nrow, 1e-3, *[t.data_ptr() for t in dev], out.data_ptr(),
                                             s.cuda_stream)
    assert rc == -1
    assert b"captured" in lib.croma_b200_last_error()
