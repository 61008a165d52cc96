"""Device chain-mesh sort vs the oracle's restatement of the reference's
recursive partition (src/chainmesh.cpp:168-213, src/particles.cpp:414-444):
bit-exact permuted arrays and cell offsets (PARITY order), identical
offsets and stable in-cell order (FAST order)."""
import numpy as np
import pytest

import oracle as O
from helpers import oracle_particles, particle_set, with_random_motion
from tigerpm_b200 import workloads as W
from tigerpm_b200.api import TigerPM, make_options

pytestmark = pytest.mark.gpu


def run_device(ps, C, sort="parity", grid=16):
    opts = make_options(round(ps.n ** (1 / 3)) or 1, grid, chain=C, sort=sort)
    with TigerPM(opts, max(ps.n, 1)) as t:
        t.set_particles(ps)
        t.chainmesh_create()
        arrays = t.get_particles()
        offsets = t.chainmesh_offsets()
        cells = [t.chainmesh_get((i, j, k)) for (i, j, k) in [(0, 0, 0), (C - 1, 0, 1), (-1, C, 2)]]
    return arrays, offsets, cells


def run_oracle(ps, C):
    p = oracle_particles(O, ps)
    pb, pe = O.chainmesh_sort(C, p)
    return p, pb, pe


@pytest.mark.parametrize("kind,n_side,C,seed", [
    ("uniform", 24, 3, 1), ("uniform", 32, 7, 2), ("uniform", 40, 11, 3),
    ("zeldovich", 32, 5, 4), ("halos", 32, 6, 5), ("uniform", 64, 45, 6),
])
def test_parity_order_bit_exact(kind, n_side, C, seed):
    ps = with_random_motion(particle_set(kind, n_side, seed), seed)
    (x, y, z, vx, vy, vz, r), offsets, cells = run_device(ps, C)
    p, pb, pe = run_oracle(ps, C)
    assert np.array_equal(x, p.x) and np.array_equal(y, p.y) and np.array_equal(z, p.z)
    assert np.array_equal(vx.view(np.uint32), p.vx.view(np.uint32))
    assert np.array_equal(vy.view(np.uint32), p.vy.view(np.uint32))
    assert np.array_equal(vz.view(np.uint32), p.vz.view(np.uint32))
    assert np.array_equal(r, p.rung)
    assert np.array_equal(offsets[:-1], pb) and np.array_equal(offsets[1:], pe)
    w = lambda i: i % C
    for (i, j, k), (b, e) in zip([(0, 0, 0), (C - 1, 0, 1), (-1, C, 2)], cells):
        key = (w(k) * C + w(j)) * C + w(i)
        assert (b, e) == (pb[key], pe[key])


def test_threshold_boundaries_and_edges():
    """Positions exactly at and one below every split threshold fixed32(m/C)."""
    C = 9
    thr = np.array([O.fixed32_from_double(m * (1.0 / C)) for m in range(C)], np.uint64)
    vals = np.concatenate([thr, np.maximum(thr, 1) - 1, [0, 2 ** 32 - 1]]).astype(np.uint32)
    g = W.rng(7)
    n = 3000
    ps = W.uniform(n, 7)
    for a in (ps.x, ps.y, ps.z):
        a[:] = g.choice(vals, n)
    ps = with_random_motion(ps, 7)
    (x, y, z, vx, vy, vz, r), offsets, _ = run_device(ps, C)
    p, pb, pe = run_oracle(ps, C)
    assert np.array_equal(x, p.x) and np.array_equal(y, p.y) and np.array_equal(z, p.z)
    assert np.array_equal(offsets[:-1], pb)


def test_one_cell_and_single_particle():
    C = 4
    ps = W.uniform(500, 9)
    ps.x[:] = ps.x % (2 ** 32 // C)  # all in x-cell 0
    ps.y[:] = ps.y % (2 ** 32 // C)
    ps.z[:] = ps.z % (2 ** 32 // C)
    (x, y, z, *_), offsets, _ = run_device(ps, C)
    p, pb, pe = run_oracle(ps, C)
    assert np.array_equal(x, p.x) and np.array_equal(z, p.z)
    ps1 = W.uniform(1, 10)
    (x1, *_), off1, _ = run_device(ps1, C)
    assert x1[0] == ps1.x[0] and off1[-1] == 1


def test_empty_box():
    ps = W.uniform(0, 1)
    (x, *_), offsets, _ = run_device(ps, 5)
    assert x.size == 0 and np.all(offsets == 0)


@pytest.mark.parametrize("kind,n_side,C", [("uniform", 32, 7), ("halos", 32, 5)])
def test_fast_order(kind, n_side, C):
    ps = particle_set(kind, n_side, 11)
    ps.vx[:] = np.arange(ps.n, dtype=np.float32)  # carries the input index
    (x, y, z, vx, *_), offsets, _ = run_device(ps, C, sort="fast")
    p, pb, pe = run_oracle(ps, C)
    assert np.array_equal(offsets[:-1], pb) and np.array_equal(offsets[1:], pe)
    idx = vx.astype(np.int64)
    assert np.array_equal(np.sort(idx), np.arange(ps.n))
    assert np.array_equal(x, ps.x[idx])
    for c in range(C ** 3):  # stable: ascending input index inside each cell
        seg = idx[offsets[c]:offsets[c + 1]]
        assert np.all(np.diff(seg) > 0)


def test_parity_dense_clump():
    """A dense clump (24,000 particles in one chain cell) among 40,000 uniform
    ones: deep recursion nodes far larger than the mean."""
    C = 6
    ps = W.uniform(64000, 17)
    g = W.rng(18)
    k = 24000
    for a in (ps.x, ps.y, ps.z):
        a[:k] = (g.integers(0, 2 ** 32 // C, k, dtype=np.uint64) + 2 * (2 ** 32 // C)).astype(np.uint32)
    ps = with_random_motion(ps, 17)
    (x, y, z, vx, vy, vz, r), offsets, _ = run_device(ps, C)
    p, pb, pe = run_oracle(ps, C)
    assert np.array_equal(x, p.x) and np.array_equal(y, p.y) and np.array_equal(z, p.z)
    assert np.array_equal(r, p.rung)
    assert np.array_equal(offsets[:-1], pb) and np.array_equal(offsets[1:], pe)
