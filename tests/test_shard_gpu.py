"""Target ranges and stage-by-stage stepping on one GPU: two contexts each
own half of a ring's targets and exchange their source records between
stages (host-ordered device copies; no kernel waits on another), and the
result equals the unsharded graph step."""
import numpy as np
import pytest

from oracle import oracle as O
from pawan_b200 import capi, cases, shard

pytestmark = pytest.mark.gpu


# FP64: the same per-target sums in the same order.  FP32C: rank 1's targets
# start mid-tile, so warps group targets differently and a few pairs at the
# far-regime boundary (u = 50) take the far limit on one side only; the
# difference stays far below the 1e-5 gate.
@pytest.mark.parametrize("prec,tol", [(capi.FP64, 1e-12), (capi.FP32C, 1e-6)])
@pytest.mark.parametrize("scheme", ["rk4", "rk3"])
def test_two_contexts_match_unsharded_step(gpu, prec, tol, scheme):
    w = cases.ring_gaussian(stations=10, per_section=1000, seed=2)  # 10,000 particles
    with capi.Context(precision=prec, nu=1e-4, chunks=4) as c:
        k = c.add_wake(w.n)
        c.set_particles(k, w)
        c.step(scheme, 0.005, 2)
        ref_pos, ref_alpha = c.state(k)
    bs = [shard.GpuShard(w, r, 2, precision=prec, nu=1e-4, chunks=4) for r in range(2)]
    shard.ShardedStepper(bs, shard.LocalExchange(bs)).step(scheme, 0.005, 2)
    pos, alpha = shard.gather_state(bs)
    for b in bs:
        b.close()
    assert O.rel_err(pos - w.pos, ref_pos - w.pos) < tol
    assert O.rel_err(alpha, ref_alpha) < tol


def test_target_range_rules(gpu):
    w = cases.ring_stations(stations=40)
    with capi.Context(precision=capi.FP32C, nu=1e-4) as c:
        k = c.add_wake(w.n)
        c.set_particles(k, w)
        c.solve()
        v_all, a_all = c.rates(k)
        c.set_target_range(0, 100, 300)
        with pytest.raises(capi.PgpuError, match="stage by stage"):
            c.step("rk4", 0.01, 1)
        with pytest.raises(capi.PgpuError, match="pgpu_diagnose_partial"):
            c.diagnose(0)
        with pytest.raises(capi.PgpuError):
            c.stage("rk4", 4, 0.01)
        # rates of the owned targets only, equal to the full evaluation's
        c.solve()
        v, a = c.rates(k)
        assert O.rel_err(v[100:400], v_all[100:400]) < 1e-6
        assert O.rel_err(a[100:400], a_all[100:400]) < 1e-6
        c.set_target_range(0, 0, -1)
        c.step("rk4", 0.01, 1)
        c.sync()


def test_records_view_the_source_records(gpu):
    import torch
    w = cases.ring_stations(stations=40)
    b = shard.GpuShard(w, 0, 1)
    torch.cuda.synchronize()
    P = b.P.cpu().numpy()
    assert np.allclose(P[:, :3], w.pos, rtol=0, atol=1e-6)
    assert np.allclose(P[:, 3], 0.5 * w.sigma ** 2, rtol=1e-6)
    assert np.allclose(b.Q.cpu().numpy()[:, :3], w.alpha, rtol=1e-6, atol=0)
    b.close()


# Diagnostics of a system split over contexts: the sum of the contexts'
# pgpu_diagnose_partial fields, combined, against pgpu_diagnose of the whole.
# FP64: the same pair terms, summed in another order (1e-12).  FP32C: the
# contexts' plans chunk the sources differently, which reorders FP32 group
# sums (1e-6, far below the 1e-5 gate).
@pytest.mark.parametrize("prec,tol", [(capi.FP64, 1e-12), (capi.FP32C, 1e-6)])
@pytest.mark.parametrize("world", [2, 3])
def test_sharded_diagnostics_match_unsharded(gpu, prec, tol, world):
    w = cases.ring_gaussian(stations=10, per_section=1000, seed=2)  # 10,000 particles
    with capi.Context(precision=prec, nu=1e-4, chunks=4) as c:
        k = c.add_wake(w.n)
        c.set_particles(k, w)
        c.step("rk4", 0.005, 2)
        ref, ref_vbi = c.diagnose(0)
    bs = [shard.GpuShard(w, r, world, precision=prec, nu=1e-4, chunks=4) for r in range(world)]
    shard.ShardedStepper(bs, shard.LocalExchange(bs)).step("rk4", 0.005, 2)
    got, vbi, zc = shard.diagnose_local(bs)
    for b in bs:
        b.close()
    scale = abs(ref[12])  # kinetic energy, the scale of the quantities that vanish
    err = np.abs(got - ref) / np.maximum(np.abs(ref), scale)
    assert np.all(err < tol), err
    assert np.abs(vbi - ref_vbi).max() <= tol * np.abs(ref_vbi).max()
    assert zc == got[14]


@pytest.mark.parametrize("prec,tol", [(capi.FP64, 1e-12), (capi.FP32C, 1e-6)])
def test_sharded_diagnostics_two_wakes(gpu, prec, tol):
    """Two wakes of one system (Zc from the last wake with weight, cross-wake
    pair terms) over three target ranges that cut through both wakes."""
    w1 = cases.ring_stations(stations=40, seed=3)
    w2 = cases.ring_stations(R=1.2, stations=40, z0=0.3, seed=5)
    n = w1.n + w2.n

    def ctx():
        c = capi.Context(precision=prec, nu=1e-4)
        a, b = c.add_wake(w1.n), c.add_wake(w2.n)
        c.set_particles(a, w1)
        c.set_particles(b, w2)
        return c

    with ctx() as c:
        ref, ref_vbi = c.diagnose(0)
    parts = []
    for r in range(3):
        first, count, _ = shard.partition(n, 3, r)
        with ctx() as c:
            c.set_target_range(0, first, count)
            parts.append(c.diagnose_partial(0))
    assert parts[0].shape == (2, capi.DIAG_FIELDS)
    got, vbi, zc = capi.diagnose_combine(sum(parts))
    scale = abs(ref[12])
    assert np.all(np.abs(got - ref) / np.maximum(np.abs(ref), scale) < tol)
    assert np.abs(vbi - ref_vbi).max() <= tol * np.abs(ref_vbi).max()


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("scheme", ["rk4", "rk3"])
def test_graphed_shard_step_equals_eager(gpu, scheme):
    """The CUDA-graph replay of one sharded step (stages + NCCL all-gathers,
    world size 1) advances the state exactly as the eager stage-by-stage
    step does."""
    import os
    from datetime import timedelta

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        w = cases.ring_gaussian(stations=10, per_section=1000, seed=2)
        eager = shard.GpuShard(w, 0, 1, precision=capi.FP64, nu=1e-4)
        graphed = shard.GpuShard(w, 0, 1, precision=capi.FP64, nu=1e-4)
        shard.ShardedStepper(eager, shard.DistExchange(eager)).step(scheme, 0.005, 3)
        g = shard.GraphedStepper(graphed, shard.DistExchange(graphed), scheme, 0.005)
        g.step(3)
        torch.cuda.synchronize()
        pe, ae = eager.state()
        pg, ag = graphed.state()
        g.close()
        eager.close()
        graphed.close()
        np.testing.assert_array_equal(pg, pe)
        np.testing.assert_array_equal(ag, ae)
    finally:
        dist.destroy_process_group()


# The surrogate on a sharded system: every context builds the octree of the
# whole system from its exchanged records and evaluates the work items that
# hold its own targets.  A target's arithmetic does not depend on which
# context owns it, so the sharded steps equal the unsharded surrogate steps
# (bitwise; asserted at 1e-12).
@pytest.mark.parametrize("world", [2, 3])
def test_sharded_surrogate_matches_unsharded(gpu, world):
    w = cases.leapfrog_rings(n_total=60000)
    kw = dict(tolerance=1.0, check_targets=512, leaf_size=64)
    with capi.Context(precision=capi.FP32C, nu=1e-4) as c:
        k = c.add_wake(w.n)
        c.set_particles(k, w)
        c.surrogate_enable(**kw)
        c.step("rk4", 0.005, 2)
        ref_pos, ref_alpha = c.state(k)
        ref_stats = c.surrogate_stats()
    bs = [shard.GpuShard(w, r, world, precision=capi.FP32C, nu=1e-4) for r in range(world)]
    for b in bs:
        b.ctx.surrogate_enable(**kw)
    shard.ShardedStepper(bs, shard.LocalExchange(bs)).step("rk4", 0.005, 2)
    pos, alpha = shard.gather_state(bs)
    stats = [b.ctx.surrogate_stats() for b in bs]
    for b in bs:
        b.close()
    assert ref_stats["evaluations"] == 8 and ref_stats["fallbacks"] == 0
    for st in stats:
        assert st["evaluations"] == 8 and st["fallbacks"] == 0
        assert st["max_err_vel"] < 1e-4 and st["max_err_dalpha"] < 1e-4
    assert O.rel_err(pos - w.pos, ref_pos - w.pos) < 1e-12
    assert O.rel_err(alpha, ref_alpha) < 1e-12


def test_sharded_surrogate_checks_owned_targets_and_falls_back(gpu):
    """A rank's sampled check draws from its own targets; with a tolerance no
    evaluation can meet, every evaluation falls back to the direct sum over
    the owned targets, whose rates then equal the direct evaluation's."""
    w = cases.leapfrog_rings(n_total=20000)
    with capi.Context(precision=capi.FP32C, nu=1e-4) as c:
        k = c.add_wake(w.n)
        c.set_particles(k, w)
        c.solve()
        v_all, a_all = c.rates(k)
        c.set_target_range(0, 5000, 8000)
        c.surrogate_enable(tolerance=1e-30, check_targets=256)
        c.solve()
        st = c.surrogate_stats()
        assert st["evaluations"] == 1 and st["fallbacks"] == 1
        v, a = c.rates(k)
        assert O.rel_err(v[5000:13000], v_all[5000:13000]) < 1e-6
        assert O.rel_err(a[5000:13000], a_all[5000:13000]) < 1e-6
