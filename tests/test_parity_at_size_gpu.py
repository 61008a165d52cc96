"""Parity at the sizes the benchmark runs, not only on small boxes.

* Chain-mesh sort, PARITY order, bit-exact against the oracle's restatement
  of the reference's recursive partition (src/chainmesh.cpp:168-213,
  src/particles.cpp:414-444): the 256^3 Zel'dovich box with chain mesh 64^3
  (the headline form) and 45^3 (the literal 256^3 configuration), and the
  64^3 uniform box with chain mesh 11^3 (the 64^3 configuration).  Permuted
  x/y/z/v/rung and every cell offset are compared.
* Kick at the headline form (256^3 particles, 768^3 cloud4 mesh, r_s = 2
  cells, cutoff 6 r_s, 64 particles per chain cell): device forces and
  potentials against the oracle's FP64 kick (src/kick_pme.cu:188-354) on a
  seeded 1 % sample of sink cells, given the device's potential; relative
  rms <= 1e-5.
* The 64^3 configuration (uniform, 64^3 CIC mesh, r_s 1.25 cells, cutoff
  4.5 r_s): the potential against the oracle's long-range solve and the
  kick against the oracle on every cell.
"""
import numpy as np
import pytest

import oracle as O
from helpers import kick_params, rel_rms
from tigerpm_b200 import workloads as W
from tigerpm_b200.api import GRAVITY_LONG_PME, Range, TigerPM, make_options

pytestmark = pytest.mark.gpu

HEADLINE = dict(n_side=256, grid=768, rs_cells=2.0, rcut_over_rs=6.0, assign="cloud4")
LITERAL = dict(n_side=256, grid=256, rs_cells=1.25, rcut_over_rs=4.5, assign="tsc")
C1 = dict(n_side=64, grid=64, rs_cells=1.25, rcut_over_rs=4.5, assign="cic")


def _opts(cfg, chain=None):
    return make_options(cfg["n_side"], cfg["grid"], chain=chain, rs_cells=cfg["rs_cells"],
                        rcut_over_rs=cfg["rcut_over_rs"], assign=cfg["assign"])


@pytest.fixture(scope="module")
def zel256():
    ps = W.zeldovich(256, 1, rms_cells=0.3, grid=256)
    g = W.rng(77)
    n = ps.n
    ps.vx[:] = g.normal(0, 1e-3, n).astype(np.float32)
    ps.vy[:] = g.normal(0, 1e-3, n).astype(np.float32)
    ps.vz[:] = g.normal(0, 1e-3, n).astype(np.float32)
    ps.rung[:] = g.integers(0, 4, n).astype(np.int8)
    return ps


def _sort_both(ps, opts):
    with TigerPM(opts, ps.n) as t:
        t.set_particles(ps)
        t.chainmesh_create()
        dev = t.get_particles()
        offs = t.chainmesh_offsets()
    p = O.Particles(*(np.array(a, copy=True) for a in ps.arrays()))
    pb, pe = O.chainmesh_sort(opts.chain_dim, p)
    return dev, offs, p, pb, pe


def _assert_sorted_equal(dev, offs, p, pb, pe):
    x, y, z, vx, vy, vz, r = dev
    assert np.array_equal(offs[:-1], pb) and np.array_equal(offs[1:], pe)
    assert np.array_equal(x, p.x) and np.array_equal(y, p.y) and np.array_equal(z, p.z)
    for a, b in ((vx, p.vx), (vy, p.vy), (vz, p.vz)):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(r, p.rung)


@pytest.mark.parametrize("chain", [64, 45])
def test_sort_bit_exact_256(zel256, chain):
    cfg = HEADLINE if chain == 64 else LITERAL
    opts = _opts(cfg, chain=chain)
    assert opts.chain_dim == chain
    _assert_sorted_equal(*_sort_both(zel256, opts))


def test_sort_bit_exact_c1():
    ps = W.uniform(64 ** 3, 1)
    g = W.rng(5)
    ps.vx[:] = g.normal(0, 1e-3, ps.n).astype(np.float32)
    ps.rung[:] = g.integers(0, 3, ps.n).astype(np.int8)
    opts = _opts(C1)
    assert opts.chain_dim == 11
    _assert_sorted_equal(*_sort_both(ps, opts))


def _device_kick(ps, opts):
    with TigerPM(opts, ps.n) as t:
        t.set_particles(ps)
        t.chainmesh_create()
        before = t.get_particles()
        t.gravity_long_compute(GRAVITY_LONG_PME)
        g = opts.four_dim
        phi = t.gravity_long_get_phi(Range((0, 0, 0), (g, g, g)))
        t.kick_pme_begin(0, 1.0, 0.01, False)
        t.kick_pme_end()
        after = t.get_particles()
        forces = t.get_forces()
        offs = t.chainmesh_offsets()
    return before, phi, after, forces, offs


def _oracle_kick_cells(opts, before, phi, offs, cells):
    p = O.Particles(*(np.array(a, copy=True) for a in before))
    kp = kick_params(O, opts, first_call=False, t0=0.01, precision=1)
    ogx, ogy, ogz, opot, counts, bad = O.kick_pme(kp, p, offs[:-1].copy(), offs[1:].copy(), phi,
                                                  sink_cells=cells)
    idx = np.concatenate([np.arange(offs[c], offs[c + 1]) for c in cells])
    return idx, np.stack([ogx, ogy, ogz], 1)[idx], opot[idx], p


def test_kick_headline_sampled_cells(zel256):
    opts = _opts(HEADLINE)
    assert opts.chain_dim == 64
    before, phi, after, (gx, gy, gz, pot), offs = _device_kick(zel256, opts)
    C = opts.chain_dim
    cells = np.sort(W.rng(2024).choice(C ** 3, size=C ** 3 // 100, replace=False)).astype(np.int32)
    idx, OG, OP, p = _oracle_kick_cells(opts, before, phi, offs, cells)
    assert idx.size > 100_000
    G = np.stack([gx, gy, gz], 1)[idx]
    assert rel_rms(G, OG) < 1e-5
    assert rel_rms(pot[idx], OP) < 1e-5
    same = after[6][idx] == p.rung[idx]
    assert np.mean(~same) < 1e-3
    V = np.stack(after[3:6], 1)[idx][same]
    OV = np.stack([p.vx, p.vy, p.vz], 1)[idx][same]
    assert rel_rms(V, OV) < 1e-5


def test_c1_potential_and_kick():
    ps = W.uniform(64 ** 3, 1)
    opts = _opts(C1)
    before, phi, after, (gx, gy, gz, pot), offs = _device_kick(ps, opts)
    ophi = O.gravity_long(64, C1["rs_cells"], 1, before[0], before[1], before[2], pme=1)
    assert rel_rms(phi, ophi) < 2e-6
    C = opts.chain_dim
    cells = np.arange(C ** 3, dtype=np.int32)
    idx, OG, OP, p = _oracle_kick_cells(opts, before, phi, offs, cells)
    assert idx.size == ps.n
    assert rel_rms(np.stack([gx, gy, gz], 1)[idx], OG) < 1e-5
    assert rel_rms(pot[idx], OP) < 1e-5
