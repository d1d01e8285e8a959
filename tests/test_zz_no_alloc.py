"""The allocation-free refine_fullres (sv_refine_fullres_noalloc).

Some callers cannot give this library device memory when they call it: an
engine that reserves all of its GPU memory at start-up and forbids later
allocations, or a plugin host that offers its plugins no allocator.  For
them sv_refine_fullres_noalloc keeps its scratch in a static device array
inside the library instead of a caller workspace.  This test calls it
through the C ABI and checks that its output is bit-identical (the
tolerance every refinement test here uses) to the workspace-based
sv_refine_fullres, on two calls in a row with different pairs, so stale
scratch from the first call cannot leak into the second.  It lives in its
own file, collected last, and needs nothing from the other tests.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run_both(svb, pair, d0, **kw):
    import torch
    lib = svb._lib.load()
    W, H = pair.W, pair.H
    p = svb.refine._params(**kw)
    left = torch.from_numpy(pair.left.ravel()).cuda()
    right = torch.from_numpy(pair.right.ravel()).cuda()
    disp0 = torch.from_numpy(d0).cuda()
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    # the existing entry point, with a caller workspace
    need = lib.sv_refine_workspace_size(W, H, ctypes.byref(p))
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    ref = torch.empty(W * H, dtype=torch.float64, device="cuda")
    assert lib.sv_refine_fullres(ptr(left), ptr(right), svb._lib.SV_U8, ptr(disp0), W, H,
                                 ctypes.byref(p), ptr(ref), None, ptr(ws), need, stream) == 0
    # the allocation-free one
    out = torch.full((W * H,), -7.0, dtype=torch.float64, device="cuda")
    flag = torch.full((1,), 99, dtype=torch.int32, device="cuda")
    rc = lib.sv_refine_fullres_noalloc(ptr(left), ptr(right), svb._lib.SV_U8, ptr(disp0), W, H,
                                       ctypes.byref(p), ptr(out), ptr(flag), stream)
    assert rc == 0, lib.sv_last_error()
    torch.cuda.synchronize()
    assert int(flag.item()) == 0
    return ref.cpu().numpy(), out.cpu().numpy()


def test_noalloc_matches_workspace_entry_point(svb):
    kw = dict(R=10, P1=12.0, P2=150.0, rx=4, ry=3)
    for seed, (W, H) in ((31, (160, 120)), (32, (203, 97))):
        pair = svb.synth.make_pair(seed, W, H, 2.0, 40.0)
        rng = np.random.default_rng(seed)
        d0 = pair.disp.ravel() + rng.uniform(-3.0, 3.0, W * H)
        ref, out = _run_both(svb, pair, d0, **kw)
        assert np.array_equal(ref.view(np.uint64), out.view(np.uint64)), (W, H)


SCRATCH = 16 << 20          # SV_NOALLOC_SCRATCH_BYTES


def _need(W, H, Kp=24, npaths=8, pbytes=1):
    """Scratch bytes of one call: header, band centres, two census maps,
    band costs and the path costs, each rounded up to 256 bytes."""
    up = lambda x: (x + 255) & ~255
    N = W * H
    return 256 + up(4 * N) + 2 * up(8 * N) + up(N * Kp) + up(N * Kp * npaths * pbytes)


def test_noalloc_capacity_limit(svb):
    """The largest 300-wide pair the static scratch holds at
    refine_disparity's parameters runs and matches; one more row is refused."""
    import torch
    lib = svb._lib.load()
    W = 300
    H = max(h for h in range(1, 400) if _need(W, h) <= SCRATCH)
    assert H >= 236 and _need(320, 240) > SCRATCH        # the documented bounds
    kw = dict(R=10, P1=12.0, P2=150.0, rx=4, ry=3)
    pair = svb.synth.make_pair(33, W, H, 2.0, 40.0)
    d0 = pair.disp.ravel() + np.random.default_rng(33).uniform(-3.0, 3.0, W * H)
    ref, out = _run_both(svb, pair, d0, **kw)
    assert np.array_equal(ref.view(np.uint64), out.view(np.uint64))
    p = svb.refine._params(**kw)
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    ptr = ctypes.c_void_p(buf.data_ptr())
    rc = lib.sv_refine_fullres_noalloc(ptr, ptr, svb._lib.SV_U8, ptr, W, H + 1,
                                       ctypes.byref(p), ptr, ctypes.c_void_p(flag.data_ptr()),
                                       None)
    assert rc == svb._lib.SV_ERR_SHAPE
    assert b"static scratch" in lib.sv_last_error()


def test_noalloc_reports_bad_disparity(svb):
    """A NaN disparity is reported through data_status, and data_status is
    required (it is the only channel for that report)."""
    import torch
    lib = svb._lib.load()
    W, H = 64, 48
    pair = svb.synth.make_pair(34, W, H, 2.0, 20.0)
    d0 = pair.disp.ravel().copy()
    d0[W * 10 + 7] = np.nan
    p = svb.refine._params(R=10, P1=12.0, P2=150.0, rx=4, ry=3)
    left = torch.from_numpy(pair.left.ravel()).cuda()
    right = torch.from_numpy(pair.right.ravel()).cuda()
    disp0 = torch.from_numpy(d0).cuda()
    out = torch.empty(W * H, dtype=torch.float64, device="cuda")
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = lib.sv_refine_fullres_noalloc(ptr(left), ptr(right), svb._lib.SV_U8, ptr(disp0), W, H,
                                       ctypes.byref(p), ptr(out), ptr(flag), None)
    assert rc == 0, lib.sv_last_error()
    torch.cuda.synchronize()
    assert int(flag.item()) == svb._lib.SV_ERR_DISP
    rc = lib.sv_refine_fullres_noalloc(ptr(left), ptr(right), svb._lib.SV_U8, ptr(disp0), W, H,
                                       ctypes.byref(p), ptr(out), None, None)
    assert rc == svb._lib.SV_ERR_NULL


def test_noalloc_rejects_oversize(svb):
    import torch
    lib = svb._lib.load()
    p = svb.refine._params(R=10, P1=12.0, P2=150.0, rx=4, ry=3)
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    ptr = ctypes.c_void_p(buf.data_ptr())
    rc = lib.sv_refine_fullres_noalloc(ptr, ptr, svb._lib.SV_U8, ptr, 1000, 1000,
                                       ctypes.byref(p), ptr, ctypes.c_void_p(flag.data_ptr()),
                                       None)
    assert rc == svb._lib.SV_ERR_SHAPE
    assert b"static scratch" in lib.sv_last_error()
