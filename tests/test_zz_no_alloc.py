"""lpk_band_chunk_device_static: the fan-out for callers that cannot allocate.

A host that renders from a real-time thread, or one that owns the whole
device through its own pool, cannot let the library call cudaMalloc while it
renders. The static entry point keeps its working memory in one file-scope
device array instead; these checks call it through the C ABI and compare it
with lpk_band_chunk_device, chunk after chunk (the array keeps the previous
call's contents, so the second call shows nothing stale leaks through).
This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from lipika_b200 import native as N
from lipika_b200 import pipeline as P
from tests import scenes

pytestmark = pytest.mark.gpu

IQ_RTOL = 1e-5  # the tolerance of the other GPU parity tests


def _run(entry, ctx, d, act, na, i0, n, out, flags):
    N.check(entry(ctx.h, C.byref(d), act, na, i0, n, None, None, out.data_ptr(), flags.data_ptr()), ctx.h)
    N.check(N.lib().lpk_sync(ctx.h), ctx.h)


def test_static_scratch_matches_allocating_entry_point_two_calls():
    import torch
    ctx = N.Context(0)
    prep = P.Prepared(scenes.config_c1(duration_s=4.0), ctx)
    L = N.lib()
    r, b = 0, 1  # the 2.048 MS/s band, six C/A transmitters
    d = prep.band_desc(r, b, 2026, 1)
    d.clock_mode = N.LPK_CLOCK_DEVICE_WALK  # the path that needs scratch for the walk
    act_list = prep.active(r, b)
    act = (C.c_int32 * len(act_list))(*act_list)
    n = 500_000
    for i0 in (3_000_000, 123_457):  # two calls in a row, the second earlier in the band
        ref = torch.zeros(2 * n, dtype=torch.float32, device="cuda")
        got = torch.full((2 * n,), float("nan"), dtype=torch.float32, device="cuda")
        fr = torch.zeros(len(act_list), dtype=torch.uint8, device="cuda")
        fg = torch.zeros(len(act_list), dtype=torch.uint8, device="cuda")
        _run(L.lpk_band_chunk_device, ctx, d, act, len(act_list), i0, n, ref, fr)
        _run(L.lpk_band_chunk_device_static, ctx, d, act, len(act_list), i0, n, got, fg)
        a = ref.cpu().numpy().view(np.complex64)
        g = got.cpu().numpy().view(np.complex64)
        assert np.all(np.isfinite(g))
        scale = float(np.max(np.abs(a)))
        assert scale > 0
        assert float(np.max(np.abs(g.astype(np.complex128) - a))) <= IQ_RTOL * scale
        assert fr.cpu().tolist() == fg.cpu().tolist() == [1] * len(act_list)
    prep.close()
    ctx.close()


def test_static_scratch_rejects_requests_beyond_its_limits():
    ctx = N.Context(0)
    prep = P.Prepared(scenes.config_c1(duration_s=1.0), ctx)
    d = prep.band_desc(0, 0, 2026, 0)  # 48 kS/s band on a 2.048 MS/s walk: 42.7 master samples per sample
    d.clock_mode = N.LPK_CLOCK_DEVICE_WALK
    act = (C.c_int32 * 1)(0)
    import torch
    out = torch.zeros(2 * 48_000, dtype=torch.float32, device="cuda")
    code = N.lib().lpk_band_chunk_device_static(ctx.h, C.byref(d), act, 1, 0, 48_000, None, None,
                                                out.data_ptr(), None)
    assert code == N.LPK_EINVAL  # 2.05e6 master samples > 2^20: refused before any launch
    assert b"static scratch limit" in N.lib().lpk_last_error(ctx.h)
    prep.close()
    ctx.close()
