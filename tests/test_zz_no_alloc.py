"""bh_gpu_trace_noalloc: the trace kernel with its scratch in a static array.

Callers that cannot call cudaMalloc - hosts whose GPU memory belongs to their
own allocator or fixed budget, plug-in hosts that forbid device allocation in
the render callback, real-time loops that cannot take cudaMalloc's implicit
device synchronisation - get this one entry point, which allocates nothing:
the work-queue counters, frame constants and deferred-ray list of the trace
kernel live in a file-scope device array of the library, and the caller owns
the output.  These tests call it through the C-ABI twice in a row (the second
call runs on the array the first one left behind) and hold each call to the
result of the context API (bh_gpu_trace_rays) for the same frame, within the
tolerances of the parity tests.

The file is named to be collected last, so that a run stopping at the first
failure has already run every other test; it also passes on its own.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from cases import kerr_a09_i60  # noqa: E402

from blackhole_b200 import Renderer, abi, gpu  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = {abi.PRECISION_FP64: 1e-6, abi.PRECISION_MIXED: 1e-3}


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_noalloc_trace_matches_context_api_on_two_calls(precision):
    torch = pytest.importorskip("torch")
    lib = gpu.load_library()
    # 96 x 80 at 4 samples: 30,720 rays, with captured rays (the mixed path
    # hands their plunge to binary64 through the deferred list in the array).
    cfg = kerr_a09_i60(width=96, height=80, sqrt_spp=2, precision=precision)
    n = cfg.n_rays
    assert n <= abi.NOALLOC_MAX_RAYS
    with Renderer(0) as r:
        ref = r.trace_rays(cfg)
    assert (ref["what"] == abi.HIT_HORIZON).sum() > 0
    order = abi.work_order(cfg.width, cfg.height, cfg.sqrt_spp)
    c = cfg.to_c()
    out = torch.empty(n * C.sizeof(abi.bh_trace_record), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    tol = TOL[precision]
    for call in (1, 2):
        with torch.cuda.stream(stream):
            out.fill_(0xFF)   # every record must be written by the call
        rc = lib.bh_gpu_trace_noalloc(0, C.byref(c), C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert rc == abi.OK, (call, abi.STATUS_NAMES.get(rc, rc))
        stream.synchronize()
        rec = np.frombuffer(out.cpu().numpy().tobytes(), dtype=abi.trace_record_dtype())
        got = np.empty_like(rec)
        got[order] = rec
        same = got["what"] == ref["what"]
        assert same.mean() == 1.0, (call, same.mean())
        assert np.array_equal(got["steps"], ref["steps"]), call
        assert np.array_equal(got["attempts"], ref["attempts"]), call
        scale = np.maximum(np.abs(ref["y"]), 1.0)
        assert (np.abs(got["y"] - ref["y"]) / scale).max() <= tol, call
        assert np.allclose(got["max_q"], ref["max_q"], rtol=tol, atol=1e-12), call
        assert np.allclose(got["max_norm"], ref["max_norm"], rtol=tol, atol=1e-12), call


def test_noalloc_rejects_frames_above_its_scratch():
    lib = gpu.load_library()
    cfg = kerr_a09_i60(width=300, height=300, sqrt_spp=1)   # 90,000 rays > 65,536
    c = cfg.to_c()
    buf = (C.c_char * 64)()
    rc = lib.bh_gpu_trace_noalloc(0, C.byref(c), C.cast(buf, C.c_void_p), None)
    assert rc == abi.ERR_INVALID_ARG
