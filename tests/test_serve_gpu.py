"""Served stream (tpm_serve_*): kick + drift requests on resident boxes,
admitted by an HBM budget, overlapping on the device.

The central check: every box's result is the same alone and in the mix.
With the deterministic (exact int64) deposit every kernel of a step is
independent of thread and block order, so a step that ran alone, a step
that ran while other boxes' steps shared the GPU, and the plain single-box
path (tpm_pme_step + tpm_drift on its own context) give identical bits."""
import numpy as np
import pytest

from helpers import with_random_motion
from tigerpm_b200 import _lib
from tigerpm_b200 import workloads as W
from tigerpm_b200.api import Server, TigerPM, TPMError, make_options

pytestmark = pytest.mark.gpu

DT = 2e-3


def _box(n, seed, deterministic=True):
    p = W.accurate_box_params(n)
    o = make_options(p["n_side"], p["grid"], rs_cells=p["rs_cells"], rcut_over_rs=p["rcut_over_rs"],
                     assign=p["assign"], deterministic_deposit=deterministic)
    ps = with_random_motion(W.zeldovich(n, seed, grid=n), seed)
    return o, ps


def _plain(o, ps):
    with TigerPM(o, ps.n) as t:
        t.set_particles(ps)
        t.pme_step(0, 1.0, 0.01, False)
        t.drift(DT)
        return t.get_particles()


def _same(a, b):
    for u, v in zip(a, b):
        assert np.array_equal(np.asarray(u).view(np.uint8), np.asarray(v).view(np.uint8))


def test_result_same_alone_and_in_the_mix():
    targets = [_box(n, 10 + n) for n in (16, 20, 24, 18)]
    others = [_box(n, 50 + n) for n in (28, 22, 26, 30, 17)]
    # alone: one request at a time
    alone = []
    with Server(max_slots=4) as s:
        ids = [s.add_box(o, ps) for o, ps in targets]
        for b in ids:
            r = s.wait(s.submit(b, DT, t0=0.01, first_call=False))
            assert r["status"] == 0 and r["particles"] == targets[b][1].n
            alone.append(s.box(b).get_particles())
    # in the mix: every box submitted at once, interleaved with other boxes
    with Server(max_slots=4) as s:
        tid = [s.add_box(o, ps) for o, ps in targets]
        oid = [s.add_box(o, ps) for o, ps in others]
        reqs = []
        for k in range(max(len(tid), len(oid))):
            if k < len(oid):
                reqs.append(s.submit(oid[k], DT, t0=0.01, first_call=False))
            if k < len(tid):
                reqs.append(s.submit(tid[k], DT, t0=0.01, first_call=False))
        for q in reqs:
            assert s.wait(q)["status"] == 0
        st = s.stats()
        assert st["max_concurrent_steps"] >= 2 and st["steps_done"] == len(reqs)
        mixed = [s.box(b).get_particles() for b in tid]
    for (o, ps), a, m in zip(targets, alone, mixed):
        _same(a, m)
        _same(a, _plain(o, ps))


def test_fp32_deposit_mix_within_tolerance():
    """With the default FP32 shared-memory deposit the summation order of a
    mesh point may differ between runs; results agree to FP32 rounding."""
    o, ps = _box(24, 7, deterministic=False)
    with Server(max_slots=3) as s:
        b = s.add_box(o, ps)
        s.wait(s.submit(b, DT, t0=0.01, first_call=False))
        got = s.box(b).get_particles()
    ref = _plain(o, ps)
    moved = ref[0].astype(np.int64) - ps.x.astype(np.int64)
    assert np.array_equal(got[6], ref[6]) or np.mean(got[6] != ref[6]) < 1e-3
    v = np.stack(got[3:6], 1).astype(np.float64)
    V = np.stack(ref[3:6], 1).astype(np.float64)
    assert np.sqrt(np.sum((v - V) ** 2) / np.sum(V * V)) < 1e-5
    assert moved.size == ps.n


def test_budget_admission_and_errors():
    o, ps = _box(24, 3)
    with Server(max_slots=2) as probe:
        probe.add_box(o, ps)
        st = probe.stats()
    # room for the working set and about two boxes' resident sets
    budget = st["max_working_set_bytes"] + int(2.5 * st["resident_bytes"])
    with Server(budget_bytes=budget, max_slots=2) as s:
        ids = []
        with pytest.raises(TPMError) as ei:
            for k in range(6):
                ids.append(s.add_box(o, ps))
        assert ei.value.status == _lib.TPM_ERR_BUDGET
        assert len(ids) == 2
        st = s.stats()
        assert st["resident_bytes"] + st["max_working_set_bytes"] <= budget
        reqs = [s.submit(b, DT, t0=0.01, first_call=False) for b in ids for _ in range(2)]
        for q in reqs:
            assert s.wait(q)["status"] == 0
        assert s.stats()["inflight_peak_bytes"] <= budget - st["resident_bytes"]
        with pytest.raises(TPMError):
            s.box(ids[0]).get_forces()  # no working set between steps
        with pytest.raises(TPMError):
            s.submit(99, DT)


def test_box_admitted_with_device_ic():
    """A box admitted with on-device initial conditions holds exactly what
    tpm_ic_zeldovich writes into a plain context."""
    from tigerpm_b200.api import ic_zeldovich
    n = 20
    p = W.accurate_box_params(n)
    o = make_options(n, p["grid"], rs_cells=p["rs_cells"], rcut_over_rs=p["rcut_over_rs"], assign="cloud4")
    with Server(max_slots=2) as s:
        b = s.add_box_ic(o, n, seed=77, rms_disp=0.3)
        got = s.box(b).get_particles()
        s.wait(s.submit(b, DT))
    with TigerPM(o, n ** 3) as t:
        ic_zeldovich(t, n, 77, rms_disp=0.3)
        ref = t.get_particles()
    _same(got, ref)


def test_poisson_replay_latencies():
    boxes = [_box(n, 80 + n, deterministic=False) for n in (16, 24, 32, 20)]
    g = W.rng(9)
    nreq = 24
    arrivals = np.cumsum(g.exponential(1.0 / 400.0, nreq))
    which = g.integers(0, len(boxes), nreq)
    with Server(max_slots=4) as s:
        ids = [s.add_box(o, ps) for o, ps in boxes]
        res = s.replay([ids[w] for w in which], arrivals, DT, t0=0.01, first_call=False)
    assert len(res) == nreq
    for r in res:
        assert r["status"] == 0
        assert r["latency_ms"] >= r["queue_ms"] >= 0
        assert r["device_ms"] > 0 and r["latency_ms"] + 1e-3 >= r["device_ms"]
