"""Per-scene accuracy of the split-precision fan-out against the all-FP64 path.

For every work unit of a scene, every band sample is rendered twice on the
GPU with noise off: once by the split-precision fan-out in accuracy mode
(lpk_split_accuracy: each fast-path (sample, transmitter) is also solved with
the reference-exact FP64 arithmetic, and the largest emission-delay and
carrier-phase differences are kept) and once by the all-FP64 kernel
(k_band_reference, the reference's per-sample arithmetic, src/channel/
mod.rs:49-101 and :236-268). The IQ difference of the two renders is taken
per band relative to the band's largest |IQ|. Device buffers are torch
tensors (memory only; the kernels are the library's).
"""
from __future__ import annotations

import ctypes as C

from . import native as N


def walk_bounded_chunk(desc: N.BandDesc, chunk: int) -> int:
    """Band samples per chunk such that the clock walk a chunk interpolates
    over (materialised per chunk on the single-band path) spans at most
    `chunk` master-clock samples: a band slower than its receiver's master
    rate takes proportionally shorter chunks."""
    fm = desc.clock_master_rate_hz
    if desc.clock_mode != N.LPK_CLOCK_DEVICE_WALK or not fm > desc.fs_hz:
        return chunk
    return max(4096, int(chunk * desc.fs_hz / fm))


def band_accuracy(ctx: N.Context, desc: N.BandDesc, active, n_samples: int, chunk: int = 1 << 24,
                  bufs=None) -> dict:
    """Accuracy triple of one band: {'delay_s', 'phase_rad', 'iq_rel', 'n_fast', 'n_exact'}.
    desc is copied; its solver is set per render and its noise turned off."""
    import torch

    L = N.lib()
    d = N.BandDesc()
    C.memmove(C.byref(d), C.byref(desc), C.sizeof(N.BandDesc))
    d.noise_power_w = 0.0
    act = (C.c_int32 * max(len(active), 1))(*active)
    dev = torch.device("cuda", ctx.device)
    if bufs is None:
        bufs = (torch.empty(2 * chunk, dtype=torch.float32, device=dev),
                torch.empty(2 * chunk, dtype=torch.float32, device=dev))
    spl, ref = bufs
    worst_d = worst_p = 0.0
    n_fast = n_exact = 0
    max_diff = torch.zeros((), dtype=torch.float64, device=dev)
    max_ref = torch.zeros((), dtype=torch.float64, device=dev)
    dd, dp = C.c_double(), C.c_double()
    nf, ne = C.c_int64(), C.c_int64()
    for i0 in range(0, n_samples, chunk):
        m = min(chunk, n_samples - i0)
        d.solver = N.LPK_SOLVER_SPLIT
        ctx.check(L.lpk_split_accuracy(ctx.h, C.byref(d), act, len(active), i0, m, None, spl.data_ptr(),
                                       C.byref(dd), C.byref(dp), C.byref(nf), C.byref(ne)))
        worst_d, worst_p = max(worst_d, dd.value), max(worst_p, dp.value)
        n_fast += nf.value
        n_exact += ne.value
        d.solver = N.LPK_SOLVER_REFERENCE
        ctx.check(L.lpk_band_chunk_device(ctx.h, C.byref(d), act, len(active), i0, m, None, None, ref.data_ptr(),
                                          None))
        stream = torch.cuda.ExternalStream(L.lpk_ctx_stream(ctx.h), device=dev)
        with torch.cuda.stream(stream):
            a = spl[:2 * m].view(m, 2).double()
            r = ref[:2 * m].view(m, 2).double()
            max_diff = torch.maximum(max_diff, torch.linalg.vector_norm(a - r, dim=1).max())
            max_ref = torch.maximum(max_ref, torch.linalg.vector_norm(r, dim=1).max())
        stream.synchronize()
    scale = float(max_ref)
    return {"delay_s": worst_d, "phase_rad": worst_p, "iq_rel": float(max_diff) / scale if scale > 0 else 0.0,
            "n_fast": n_fast, "n_exact": n_exact}


def scene_accuracy(ctx: N.Context, prep, seed: int = 2026, chunk: int = 1 << 24) -> dict:
    """The accuracy triple of a whole scene: the largest delay error (ps),
    carrier-phase error (rad) and per-band IQ error (relative to the band's
    max |IQ|) over every work unit, with the clock walk generated on the
    device (the headline path's clock) and noise off."""
    import torch

    dev = torch.device("cuda", ctx.device)
    bufs = (torch.empty(2 * chunk, dtype=torch.float32, device=dev),
            torch.empty(2 * chunk, dtype=torch.float32, device=dev))
    out = {"delay_ps": 0.0, "phase_rad": 0.0, "iq_rel": 0.0, "txrx_fast": 0, "txrx_exact": 0, "units": 0}
    for w, (r, b) in enumerate(prep.work()):
        d = prep.band_desc(r, b, seed, w)
        if d.clock_mode == N.LPK_CLOCK_HOST:
            d.clock_mode = N.LPK_CLOCK_DEVICE_WALK
        res = band_accuracy(ctx, d, prep.active(r, b), prep.n_samples(r, b), walk_bounded_chunk(d, chunk), bufs)
        out["delay_ps"] = max(out["delay_ps"], 1e12 * res["delay_s"])
        out["phase_rad"] = max(out["phase_rad"], res["phase_rad"])
        out["iq_rel"] = max(out["iq_rel"], res["iq_rel"])
        out["txrx_fast"] += res["n_fast"]
        out["txrx_exact"] += res["n_exact"]
        out["units"] += 1
    return out
