"""Batched ensemble (tpm_batch_*): many independent boxes kicked together.

Each box's result in the batch -- sorted particles, forces, potentials,
velocities and rungs after one PME kick -- is compared with the same box
kicked alone through the plain single-box path (tpm_pme_step on its own
context).  The chain-mesh order of every box is bit-exact against the
oracle's restatement of the reference partition (src/chainmesh.cpp:168-213).
Graph replays are compared with the eager step bit for bit when the deposit
is deterministic, and the autotuner must leave velocities and rungs as they
were."""
import numpy as np
import pytest

import oracle as O
from helpers import rel_rms, with_random_motion
from tigerpm_b200 import workloads as W
from tigerpm_b200.api import Batch, TigerPM, make_options

pytestmark = pytest.mark.gpu


def _boxes(sides, seed, deterministic=False):
    opts, sets = [], []
    for i, n in enumerate(sides):
        p = W.accurate_box_params(int(n))
        opts.append(make_options(p["n_side"], p["grid"], rs_cells=p["rs_cells"], rcut_over_rs=p["rcut_over_rs"],
                                 assign=p["assign"], deterministic_deposit=deterministic))
        sets.append(with_random_motion(W.zeldovich(int(n), seed + i, grid=int(n)), seed + i))
    return opts, sets


def _solo(opts, ps, first_call=False, t0=0.01):
    with TigerPM(opts, ps.n) as t:
        t.set_particles(ps)
        t.pme_step(0, 1.0, t0, first_call)
        t.check_errors()
        return t.get_particles(), t.get_forces()


def _batch_results(b, i):
    t = b.box(i)
    return t.get_particles(), t.get_forces()


def _compare(res, ref, tol=1e-5):
    (x, y, z, vx, vy, vz, r), (gx, gy, gz, pot) = res
    (X, Y, Z, VX, VY, VZ, R), (GX, GY, GZ, POT) = ref
    assert np.array_equal(x, X) and np.array_equal(y, Y) and np.array_equal(z, Z)
    assert rel_rms(np.stack([gx, gy, gz], 1), np.stack([GX, GY, GZ], 1)) < tol
    assert rel_rms(pot, POT) < tol
    same = r == R
    assert np.mean(~same) < 2e-3
    assert rel_rms(np.stack([vx, vy, vz], 1)[same], np.stack([VX, VY, VZ], 1)[same]) < tol


@pytest.mark.parametrize("graph", [False, True])
def test_batch_matches_solo_boxes(graph):
    sides = [16, 20, 24, 17, 28, 32]
    opts, sets = _boxes(sides, 100)
    with Batch(opts, [s.n for s in sets]) as b:
        for i, ps in enumerate(sets):
            b.set_input(i, ps)
        b.step(restore=True, graph=graph, t0=0.01, first_call=False)
        b.synchronize()
        for i in range(len(sides)):
            b.box(i).check_errors()
            _compare(_batch_results(b, i), _solo(opts[i], sets[i]))
            # chain-mesh order: bit-exact against the oracle
            p = O.Particles(*(np.array(a, copy=True) for a in sets[i].arrays()))
            pb, pe = O.chainmesh_sort(opts[i].chain_dim, p)
            offs = b.box(i).chainmesh_offsets()
            assert np.array_equal(offs[:-1], pb) and np.array_equal(offs[1:], pe)


def test_graph_replay_bit_exact_and_sequential_path():
    """With the deterministic deposit every kernel of a step is order
    independent: eager step, first graph replay, second graph replay and the
    box-after-box plain path all give the same bits."""
    sides = [20, 24, 16, 30]
    opts, sets = _boxes(sides, 200, deterministic=True)
    with Batch(opts, [s.n for s in sets]) as b:
        for i, ps in enumerate(sets):
            b.set_input(i, ps)
        runs = []
        for mode in ("eager", "graph", "graph", "sequential"):
            if mode == "sequential":
                b.steps_sequential(restore=True, t0=0.01, first_call=False)
            else:
                b.step(restore=True, graph=(mode == "graph"), t0=0.01, first_call=False)
            b.synchronize()
            runs.append([_batch_results(b, i) for i in range(len(sides))])
        for i in range(len(sides)):
            base = runs[0][i]
            for k in (1, 2):
                for a, c in zip(base[0] + base[1], runs[k][i][0] + runs[k][i][1]):
                    assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(c).view(np.uint8))
            _compare(runs[3][i], base)


def test_autotune_restores_state_and_picks_valid_shape():
    sides = [24, 20, 28]
    opts, sets = _boxes(sides, 300)
    with Batch(opts, [s.n for s in sets]) as b:
        for i, ps in enumerate(sets):
            b.set_input(i, ps)
        b.step(restore=True, graph=False, t0=0.01, first_call=False)
        b.synchronize()
        before = [b.box(i).get_particles() for i in range(len(sides))]
        best = b.autotune(repeats=1)
        assert best["tuned"] == 1 and best["ms"] > 0
        assert best["warps"] in (2, 4, 8) and best["npass"] & (best["npass"] - 1) == 0
        after = [b.box(i).get_particles() for i in range(len(sides))]
        for u, v in zip(before, after):
            for a, c in zip(u, v):
                assert np.array_equal(a, c)
        assert b.shape()["warps"] == best["warps"]
        # the tuned shape gives the same kick as the solo path
        b.step(restore=True, graph=True, t0=0.01, first_call=False)
        b.synchronize()
        for i in range(len(sides)):
            _compare(_batch_results(b, i), _solo(opts[i], sets[i]))


def test_batch_with_wrapping_box():
    """A box whose chain mesh is 3 cells wide takes the minimum-image form of
    the pair kernel; the whole batch then runs it."""
    o_small = make_options(12, 36, chain=3, rs_cells=2.0, rcut_over_rs=6.0)
    o_big = make_options(24, 72, rs_cells=2.0, rcut_over_rs=6.0)
    sets = [with_random_motion(W.uniform(12 ** 3, 5), 5), with_random_motion(W.uniform(24 ** 3, 6), 6)]
    opts = [o_small, o_big]
    with Batch(opts, [s.n for s in sets]) as b:
        for i, ps in enumerate(sets):
            b.set_input(i, ps)
        b.step(restore=True, graph=True, t0=0.01, first_call=False)
        b.synchronize()
        for i in range(2):
            _compare(_batch_results(b, i), _solo(opts[i], sets[i]))


def test_batch_errors():
    o = make_options(16, 48, rs_cells=2.0, rcut_over_rs=6.0)
    with Batch([o], [4096]) as b:
        with pytest.raises(Exception):
            b.set_input(3, W.uniform(100, 1))
        with pytest.raises(Exception):
            b.set_shape(3, 100, 48)  # stage not a multiple of 128, npass not a power of two
        with pytest.raises(Exception):
            b.autotune()  # needs a completed step
