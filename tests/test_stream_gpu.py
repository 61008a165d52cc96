"""Served stream (tpm_pme_steps_host): several boxes host -> device -> host
with the transfers overlapped; every step must give exactly what the
sequential set_particles / pme_step / get_particles calls give for the same
box (exact deposit, so the whole step is bit-reproducible)."""
import numpy as np
import pytest

from helpers import particle_set, with_random_motion
from tigerpm_b200 import workloads as W
from tigerpm_b200.api import TigerPM, make_options

pytestmark = pytest.mark.gpu


def pinned_like(ps):
    torch = pytest.importorskip("torch")
    ts = [torch.from_numpy(np.array(a, copy=True)).pin_memory() for a in ps.arrays()]
    return ts, W.ParticleSet(*(t.numpy() for t in ts))


def empty_like(ps):
    return W.ParticleSet(*(np.empty_like(a) for a in ps.arrays()))


def sequential(opts, boxes, **kw):
    out = []
    with TigerPM(opts, boxes[0].n) as t:
        for b in boxes:
            t.set_particles(b)
            t.pme_step(**kw)
            out.append(t.get_particles())
    return out


@pytest.mark.parametrize("grid,fft", [(48, "auto"), (40, "cufft")])
def test_stream_matches_sequential_steps(grid, fft):
    boxes = [with_random_motion(particle_set(k, 20, 30 + i, grid), 30 + i, max_rung=3)
             for i, k in enumerate(["uniform", "zeldovich", "halos", "uniform", "zeldovich"])]
    opts = make_options(20, grid, rs_cells=1.5, rcut_over_rs=4.0, deterministic_deposit=True, fft=fft)
    kw = dict(min_rung=1, scale=1.0, t0=0.5, first_call=False)
    ref = sequential(opts, boxes, **kw)
    keep = [pinned_like(b) for b in boxes]
    ins = [p for _, p in keep]
    outs = [empty_like(b) for b in boxes]
    with TigerPM(opts, boxes[0].n) as t:
        t.pme_steps_host(ins, outs, **kw)
        last = t.get_particles()
        # a second call on the same context, every step into one output set
        shared = empty_like(boxes[0])
        t.pme_steps_host(ins[:3], [shared] * 3, **kw)
    for o, r in zip(outs, ref):
        for a, b in zip(o.arrays(), r):
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    for a, b in zip(last, ref[-1]):
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    for a, b in zip(shared.arrays(), ref[2]):
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_stream_single_step_and_empty():
    box = particle_set("uniform", 16, 7)
    opts = make_options(16, 32, rs_cells=1.5, rcut_over_rs=4.0, deterministic_deposit=True)
    ref = sequential(opts, [box], min_rung=0)
    out = empty_like(box)
    with TigerPM(opts, box.n) as t:
        t.pme_steps_host([], [])
        t.pme_steps_host([box], [out], min_rung=0)
    for a, b in zip(out.arrays(), ref[0]):
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
