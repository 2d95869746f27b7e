"""lpk_band_chunk_device_static: the fan-out for callers that cannot allocate.

A host that renders from a real-time thread, or one that owns the whole
device through its own pool, cannot let the library call cudaMalloc while it
renders. The static entry point keeps its working memory in one file-scope
device array instead; these checks call it through the C ABI and compare it
with lpk_band_chunk_device, chunk after chunk, for both solvers, with a
flicker clock, with an orbiting receiver and with an antenna (the array keeps the previous call's contents, so the second call
shows nothing stale leaks through), and time the walk rebuild it does on
every call.
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


def _compare_two_calls(ctx, prep, d, r, b, n, starts, expect_flags=None):
    """Both entry points on the same chunks, one call after the other; the
    static one must give the allocating one's bits (same kernels, same
    inputs) and never anything stale from the call before."""
    import torch
    L = N.lib()
    act_list = prep.active(r, b)
    act = (C.c_int32 * len(act_list))(*act_list)
    for i0 in starts:
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
        assert np.array_equal(a, g), (i0, d.solver)
        assert fr.cpu().tolist() == fg.cpu().tolist()
        if expect_flags is not None:
            assert fg.cpu().tolist() == expect_flags(len(act_list))


def test_static_scratch_matches_allocating_entry_point_two_calls():
    ctx = N.Context(0)
    prep = P.Prepared(scenes.config_c1(duration_s=4.0), ctx)
    r, b = 0, 1  # the 2.048 MS/s band, six C/A transmitters
    d = prep.band_desc(r, b, 2026, 1)
    d.clock_mode = N.LPK_CLOCK_DEVICE_WALK  # the path that needs scratch for the walk
    for solver in (N.LPK_SOLVER_REFERENCE, N.LPK_SOLVER_SPLIT):
        d.solver = solver
        # two calls in a row, the second earlier in the band
        _compare_two_calls(ctx, prep, d, r, b, 500_000, (3_000_000, 123_457), lambda k: [1] * k)
    prep.close()
    ctx.close()


def test_static_scratch_flicker_clock_both_solvers():
    """A receiver clock with a white-FM walk and a flicker floor: the static
    entry point stages the chunk's flicker points in its array too."""
    from lipika_b200 import config as cfg
    ctx = N.Context(0)
    clock = cfg.Clock(allan_deviation_1s=1e-11, flicker_floor=3e-10, frequency_offset_y0=0.4e-6)
    prep = P.Prepared(scenes.config_c1(duration_s=3.0, clock=clock), ctx)
    d = prep.band_desc(0, 1, 2026, 1)
    d.clock_mode = N.LPK_CLOCK_DEVICE_WALK
    assert d.flicker_n > 0
    for solver in (N.LPK_SOLVER_REFERENCE, N.LPK_SOLVER_SPLIT):
        d.solver = solver
        _compare_two_calls(ctx, prep, d, 0, 1, 400_000, (2_000_000, 77_777), lambda k: [1] * k)
    prep.close()
    ctx.close()


def test_static_scratch_orbiting_receiver_both_solvers():
    """A receiver on a circular Keplerian orbit (positions on the device)."""
    from lipika_b200 import workloads as W
    ctx = N.Context(0)
    sc = scenes.config_c1(duration_s=2.0)
    sc.receivers[0].trajectory = W._kepler(6_900_000.0, 60.0, 30.0, 100.0)
    prep = P.Prepared(sc, ctx)
    d = prep.band_desc(0, 1, 2026, 1)
    d.clock_mode = N.LPK_CLOCK_DEVICE_WALK
    assert d.rx_kind == N.LPK_RX_KEPLER
    for solver in (N.LPK_SOLVER_REFERENCE, N.LPK_SOLVER_SPLIT):
        d.solver = solver
        _compare_two_calls(ctx, prep, d, 0, 1, 300_000, (1_500_000, 31_337), lambda k: [1] * k)
    prep.close()
    ctx.close()


def test_static_scratch_antenna_band_both_solvers():
    """A band with an antenna (per-transmitter occlusion flags from the
    kernel) over a 64-transmitter sky, both solvers."""
    from lipika_b200 import config as cfg
    ctx = N.Context(0)
    sc = scenes.config_c4(duration_s=2.0, n_rx=1, noise=False)
    sc.receivers[0].bands[0].frontend = cfg.Frontend(
        antenna={"peak_dbi": 3.9, "horizon_dbi": -3.0, "fb_db": 8.5, "cutoff_deg": 10.0})
    prep = P.Prepared(sc, ctx)
    d = prep.band_desc(0, 0, 2026, 0)
    d.clock_mode = N.LPK_CLOCK_DEVICE_WALK
    assert d.has_antenna
    for solver in (N.LPK_SOLVER_REFERENCE, N.LPK_SOLVER_SPLIT):
        d.solver = solver
        _compare_two_calls(ctx, prep, d, 0, 0, 200_000, (1_000_000, 0))
    prep.close()
    ctx.close()


def test_static_scratch_walk_cost_grows_with_offset():
    """Every call rebuilds the walk from master sample 0: one chunk near the
    end of a 120 s band costs more than the same chunk at its start."""
    import torch
    ctx = N.Context(0)
    prep = P.Prepared(scenes.config_c1(duration_s=120.0), ctx)
    L = N.lib()
    d = prep.band_desc(0, 1, 2026, 1)
    d.clock_mode = N.LPK_CLOCK_DEVICE_WALK
    d.solver = N.LPK_SOLVER_SPLIT
    act_list = prep.active(0, 1)
    act = (C.c_int32 * len(act_list))(*act_list)
    n = 1 << 19
    out = torch.zeros(2 * n, dtype=torch.float32, device="cuda")
    stream = torch.cuda.ExternalStream(L.lpk_ctx_stream(ctx.h))
    ms = {}
    for i0 in (0, 118 * 2_048_000):
        for rep in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            N.check(L.lpk_band_chunk_device_static(ctx.h, C.byref(d), act, len(act_list), i0, n, None, None,
                                                   out.data_ptr(), None), ctx.h)
            e1.record(stream)
            e1.synchronize()
            ms[i0] = e0.elapsed_time(e1)
    print(f"static entry point, 2^19 samples x 6 transmitters: {ms[0]:.3f} ms at 0 s, "
          f"{ms[118 * 2_048_000]:.3f} ms at 118 s")
    assert ms[118 * 2_048_000] > ms[0]
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
