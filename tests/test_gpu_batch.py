"""The batched fan-out (lpk_batch_*, lpk_generate_scene) against the
single-band entry points on the same scenes and seeds.

The batch renders every (receiver, band) work unit in rounds of equal time;
its outputs must not depend on that: with the reference solver they equal
lpk_band_chunk bit for bit (same exact arithmetic, same walk values from
the shared per-receiver walk), with the split solver they equal the
single-band split kernel of the same launch shape, and any round length or
round order gives the same bits.
"""
import ctypes as C

import numpy as np
import pytest

from lipika_b200 import native as N
from lipika_b200 import pipeline as P
from tests import scenes

pytestmark = pytest.mark.gpu

SPLIT_RTOL = 1e-6  # batch vs single-band split kernel, x max|single|


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


def _units(prep, solver, clock_mode=N.LPK_CLOCK_DEVICE_WALK, noise=True, seed=2026):
    units = []
    for w, (r, b) in enumerate(prep.work()):
        d = prep.band_desc(r, b, seed, w)
        d.solver = solver
        d.clock_mode = clock_mode
        if not noise:
            d.noise_power_w = 0.0
        units.append((d, prep.active(r, b), prep.n_samples(r, b)))
    return units


def _single(ctx, units, variant=0):
    ctx.check(N.lib().lpk_ctx_set_split_variant(ctx.h, variant))
    outs = []
    for d, act, n in units:
        out = np.zeros(max(n, 1), np.complex64)
        a = np.ascontiguousarray(np.asarray(act, np.int32))
        ctx.check(N.lib().lpk_band_chunk(ctx.h, C.byref(d), a.ctypes.data_as(N._I32) if a.size else None, a.size,
                                         0, n, None, None, out.ctypes.data_as(N._CF), None))
        outs.append(out[:n])
    ctx.check(N.lib().lpk_ctx_set_split_variant(ctx.h, 0))
    return outs


def _rel(a, b):
    scale = max(float(np.max(np.abs(b))) if b.size else 0.0, 1e-30)
    return float(np.max(np.abs(a.astype(np.complex128) - b))) / scale if b.size else 0.0


def _uneven_scene():
    # 3 receivers with 1-3 bands of 48 kS/s - 4.096 MS/s, 24 C/A transmitters
    return scenes.config_c2(duration_s=0.6, n_rx=3)


def test_batch_reference_solver_is_bit_exact(ctx):
    prep = P.Prepared(_uneven_scene(), ctx)
    units = _units(prep, N.LPK_SOLVER_REFERENCE)
    single = _single(ctx, units)
    b = N.Batch(ctx, units, round_s=0.25)
    got = b.render()
    for u, (x, y) in enumerate(zip(got, single)):
        assert x.shape == y.shape, u
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), (u, _rel(x, y))
    b.close()
    prep.close()


@pytest.mark.parametrize("variant", range(6))
def test_batch_split_matches_single_band(ctx, variant):
    prep = P.Prepared(scenes.config_c1(duration_s=1.5), ctx)
    units = _units(prep, N.LPK_SOLVER_SPLIT)
    prep2 = P.Prepared(_uneven_scene(), ctx)
    units2 = _units(prep2, N.LPK_SOLVER_SPLIT)
    for us in (units, units2):
        single = _single(ctx, us, variant)
        b = N.Batch(ctx, us, round_s=0.4)
        b.set_config(variant)
        got = b.render()
        exact = 0
        for u, (x, y) in enumerate(zip(got, single)):
            assert x.shape == y.shape
            assert _rel(x, y) <= SPLIT_RTOL, (variant, u, _rel(x, y))
            exact += int(np.array_equal(x.view(np.uint32), y.view(np.uint32)))
        print(f"variant {variant}: {exact}/{len(got)} units bit-identical to the single-band kernel")
        b.close()
    prep.close()
    prep2.close()


def test_batch_noise_only_and_empty_units(ctx):
    """A band no transmitter falls in (noise and the receiver chain only)
    and a unit of zero length ride along in a batch: the first matches the
    single-band kernel, the second yields nothing, and neither disturbs the
    other units."""
    prep = P.Prepared(_uneven_scene(), ctx)
    for solver in (N.LPK_SOLVER_REFERENCE, N.LPK_SOLVER_SPLIT):
        units = _units(prep, solver)
        d0, _, n0 = units[0]
        quiet = type(d0).from_buffer_copy(d0)
        quiet.noise_seed = d0.noise_seed + 1000
        empty = type(units[1][0]).from_buffer_copy(units[1][0])
        units = units + [(quiet, [], n0), (empty, units[1][1], 0)]
        single = _single(ctx, units[:-1]) + [np.zeros(0, np.complex64)]
        b = N.Batch(ctx, units, round_s=0.25)
        got = b.render()
        b.close()
        for u, (x, y) in enumerate(zip(got, single)):
            assert x.shape == y.shape, (solver, u)
            if solver == N.LPK_SOLVER_REFERENCE or u >= len(units) - 2:
                assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), (solver, u, _rel(x, y))
            else:
                assert _rel(x, y) <= SPLIT_RTOL, (solver, u, _rel(x, y))
        assert got[-2].size == n0 and np.any(got[-2] != 0)  # noise only
    prep.close()


def test_batch_with_256_transmitters_in_a_band(ctx):
    """The most in-band transmitters a band takes (256): their tables and
    anchor records staged in ~156 KB of shared memory (one fan-out block per
    SM). Batch, single-band split kernel and the FP64 kernel agree."""
    sc = scenes.config_c4(duration_s=0.05, n_rx=1, n_tx=256, noise=False)
    prep = P.Prepared(sc, ctx)
    assert [len(prep.active(r, b)) for (r, b) in prep.work()] == [256]
    units = _units(prep, N.LPK_SOLVER_SPLIT)
    split = _single(ctx, units)
    ref = _single(ctx, _units(prep, N.LPK_SOLVER_REFERENCE))
    b = N.Batch(ctx, units, round_s=0.02)
    got = b.render()
    v, bps, mx = b.config()
    b.close()
    print(f"256 transmitters: {bps} fan-out block(s) per SM (of {mx})")
    assert _rel(got[0], split[0]) <= SPLIT_RTOL
    assert _rel(got[0], ref[0]) <= 1e-5
    prep.close()


def test_batch_round_length_and_order_do_not_change_bits(ctx):
    prep = P.Prepared(_uneven_scene(), ctx)
    units = _units(prep, N.LPK_SOLVER_SPLIT)
    ref = N.Batch(ctx, units, round_s=1.0).render()
    b = N.Batch(ctx, units, round_s=0.13)
    parts = [[None] * b.n_rounds for _ in units]
    for r in reversed(range(b.n_rounds)):  # late rounds first: carries are completed on the way
        b.run(r)
        for u in range(len(units)):
            n = b.extent(r, u)[1]
            if n > 0:
                parts[u][r] = b.output(u)[:n].copy()
    for u in range(len(units)):
        got = np.concatenate([p for p in parts[u] if p is not None])
        assert np.array_equal(got.view(np.uint32), ref[u].view(np.uint32)), u
    prep.close()


def test_batch_deterministic_clock_and_no_walk(ctx):
    prep = P.Prepared(scenes.config_c1(duration_s=1.0), ctx)
    units = _units(prep, N.LPK_SOLVER_REFERENCE, clock_mode=N.LPK_CLOCK_DETERMINISTIC, noise=False)
    single = _single(ctx, units)
    got = N.Batch(ctx, units, round_s=0.3).render()
    for x, y in zip(got, single):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    prep.close()


def test_batch_autotune_picks_a_measured_shape(ctx):
    prep = P.Prepared(_uneven_scene(), ctx)
    units = _units(prep, N.LPK_SOLVER_SPLIT)
    b = N.Batch(ctx, units, round_s=0.3)
    tab = b.autotune(rnd=1, reps=2)
    measured = tab[tab > 0]
    assert measured.size >= len(N.split_variants())
    v, bps, max_bps = b.config()
    assert 1 <= bps <= max_bps
    assert abs(tab[v, 0 if bps == max_bps else 1] - measured.min()) < 1e-9
    print("autotune ms per round (variant x [max, half] blocks/SM):\n", tab, "-> variant", v, "bps", bps)
    single = _single(ctx, units, v)
    got = b.render()
    for x, y in zip(got, single):
        assert _rel(x, y) <= SPLIT_RTOL
    prep.close()


def test_generate_scene_matches_generate_band(ctx):
    sc = _uneven_scene()
    prep = P.Prepared(sc, ctx)
    work = prep.work()
    batched = {w: [] for w in range(len(work))}
    prep.generate_scene(2026, 0.2, lambda w, c: batched[w].append(c) and False, noise=True,
                        device_clock=True, split=True)
    for w, (r, b) in enumerate(work):
        chunks = []
        prep.generate_band(r, b, 2026, w, 1 << 18, lambda c: chunks.append(c) and False, noise=True,
                           device_clock=True, split=True)
        x = np.concatenate(batched[w])
        y = np.concatenate(chunks)
        assert x.shape == y.shape
        assert _rel(x, y) <= SPLIT_RTOL, (w, _rel(x, y))
    prep.close()


def test_batch_profiling_times_each_fanout_without_changing_bits(ctx):
    prep = P.Prepared(_uneven_scene(), ctx)
    units = _units(prep, N.LPK_SOLVER_SPLIT)
    L = N.lib()
    b = N.Batch(ctx, units, round_s=0.25)
    ctx.check(L.lpk_profile_reset(ctx.h))
    ctx.check(L.lpk_profile_enable(ctx.h, 1))
    got = b.render()
    ms, fan, alln = C.c_double(), C.c_int64(), C.c_int64()
    ctx.check(L.lpk_profile_read(ctx.h, C.byref(ms), C.byref(fan), C.byref(alln)))
    ctx.check(L.lpk_profile_enable(ctx.h, 0))
    assert fan.value == b.n_rounds  # one timed persistent fan-out per round
    assert alln.value == 5 * b.n_rounds  # walk scan, group sums, carries, anchors, fan-out
    assert ms.value > 0.0
    ref = N.Batch(ctx, units, round_s=0.25).render()
    for x, y in zip(got, ref):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    prep.close()


def test_rank_shards_reproduce_the_whole_scene(ctx):
    """Each rank of a 2-way receiver sharding (run here one after the
    other on one GPU: the shards share nothing) renders exactly what the
    single batch over every unit renders."""
    from lipika_b200 import shard as S
    prep = P.Prepared(_uneven_scene(), ctx)
    whole = N.Batch(ctx, _units(prep, N.LPK_SOLVER_SPLIT), round_s=0.25).render()
    got = {}
    for rank in range(2):
        part = S.render_rank_gpu(prep, rank, 2, seed=2026, round_s=0.3)
        assert not set(part) & set(got)
        got.update(part)
    assert sorted(got) == list(range(len(whole)))
    for w, iq in got.items():
        assert np.array_equal(iq.view(np.uint32), whole[w].view(np.uint32)), w
    prep.close()


def test_full_scene_split_batch_matches_fp64_batch(ctx):
    """The whole 120 s dual-band scene (251.5 M band samples, 1.48e9 tx·rx
    samples), rendered by the batched fan-out twice, split and all-FP64,
    with the same device clock walk and noise off: every band sample of the
    split render within the split path's IQ bar of the FP64 render."""
    sc = scenes.config_c1(duration_s=120.0, noise=False)
    prep = P.Prepared(sc, ctx)
    outs = {}
    for solver in (N.LPK_SOLVER_REFERENCE, N.LPK_SOLVER_SPLIT):
        units = _units(prep, solver, noise=False)
        b = N.Batch(ctx, units, round_s=30.0)
        outs[solver] = b.render()
        b.close()
    worst = 0.0
    for u, (x, y) in enumerate(zip(outs[N.LPK_SOLVER_SPLIT], outs[N.LPK_SOLVER_REFERENCE])):
        assert x.shape == y.shape == (prep.n_samples(*prep.work()[u]),)
        r = _rel(x, y)
        worst = max(worst, r)
        assert r <= 1e-5, (u, r)
    print(f"full 120 s scene, batched split vs batched FP64: worst IQ error {worst:.2e} of max")
    prep.close()


def test_scene_to_dir_through_the_batch(ctx, tmp_path):
    """run_scene_to_dir on the batch (lpk_generate_scene_to_files): each
    band's .iq.c64 holds exactly what lpk_generate_scene hands its sink, and
    every band has its sidecar."""
    sc = scenes.config_c1(duration_s=3.0)
    man = P.run_scene_to_dir(sc, 4242, str(tmp_path), ctx=ctx, device_clock=True, round_s=1.0)
    prep = P.Prepared(sc, ctx)
    got = {}
    prep.generate_scene(4242, 1.0, lambda w, c: got.setdefault(w, []).append(c) and False)
    assert len(man) == len(prep.work()) == len(got)
    for w, m in enumerate(man):
        data = np.fromfile(m.path, dtype=np.complex64)
        assert data.size == m.n_samples == prep.n_samples(*prep.work()[w]) > 0
        assert data.tobytes() == np.concatenate(got[w]).tobytes()
        assert (tmp_path / f"{m.name}.iq.json").exists()
    prep.close()
