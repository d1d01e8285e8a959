"""Failure detection without a GPU fault: the bounded waits give up and
report SV_ERR_TIMEOUT, and the CUDA context stays usable afterwards.

The device wait is the one every tcgen05 convolution uses (an mbarrier the
MMA commit arrives at): here nothing arrives, the poll count runs out, the
kernel records the timeout, frees its tensor memory and returns.  The host
wait is predict_auto's poll of the mapped slot a stage publishes its peak
into: here no stage runs, the stream is idle, and the poll returns an error
instead of spinning."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_device_wait_times_out_and_frees(svb):
    import torch
    lib = svb._lib.load()
    fd = torch.zeros(2, dtype=torch.int32, device="cuda")
    rc = lib.sv_selftest_wait_timeout(4096, ctypes.c_void_p(fd.data_ptr()), None)
    assert rc == svb._lib.SV_OK, lib.sv_last_error()
    torch.cuda.synchronize()
    flag, done = fd.cpu().tolist()
    assert flag == svb._lib.SV_ERR_TIMEOUT and done == 1
    # the context is intact: tensor memory was released (a second CTA can
    # allocate it) and ordinary work still runs
    fd.zero_()
    assert lib.sv_selftest_wait_timeout(64, ctypes.c_void_p(fd.data_ptr()), None) == 0
    torch.cuda.synchronize()
    assert fd.cpu().tolist() == [svb._lib.SV_ERR_TIMEOUT, 1]
    pair = svb.synth.make_pair(3, 64, 48, 2.0, 20.0)
    out, st = svb.refine.lr_refine(pair.left, pair.right, pair.disp.ravel(), 64, 48, tol=2.0,
                                   R=10, P1=12.0, P2=150.0, rx=4, ry=3)
    assert np.isfinite(out).all()


def test_host_slot_poll_times_out(svb):
    import torch
    lib = svb._lib.load()
    s = torch.cuda.Stream()
    rc = lib.sv_selftest_slot_wait(ctypes.c_void_p(s.cuda_stream))
    assert rc == svb._lib.SV_ERR_TIMEOUT
    assert b"not written" in lib.sv_last_error()
