"""Strongly clustered boxes: one chain cell holding hundreds of times the
mean occupancy (the NFW-halo configuration in miniature).

The default kick takes (cell, sink pass) work items from a cost-sorted
queue, so a heavy cell is spread over many blocks instead of one block per
cell (the reference's static contiguous cell split per block,
src/kick_pme.cu:139-141, leaves such a cell on one block).  Each pass item
streams the whole neighbourhood with the same staging as the per-cell
launch, so the two launch forms agree bit for bit; both agree with the
oracle's FP64 kick (src/kick_pme.cu:188-354) on the heavy cell and on a
sample of ordinary cells."""
import numpy as np
import pytest

import oracle as O
from helpers import kick_params, rel_rms, with_random_motion
from tigerpm_b200 import workloads as W
from tigerpm_b200.api import GRAVITY_LONG_PME, Range, TigerPM, make_options

pytestmark = pytest.mark.gpu


def clumped(n_side, clump, seed):
    """n_side^3 particles: `clump` of them in a Gaussian blob of 0.05 chain
    cells around a chain-cell centre, the rest uniform."""
    ps = W.uniform(n_side ** 3, seed)
    g = W.rng(seed + 1)
    C = n_side // 4  # chain cells per side of the accurate form
    centre = (np.array([2, 7, 4]) + 0.5) / C  # a cell centre
    pos = centre[:, None] + g.normal(0, 0.05 / (n_side / 4), (3, clump))
    raw = np.floor(np.mod(pos, 1.0) * 2.0 ** 32).astype(np.uint64).astype(np.uint32)
    ps.x[:clump], ps.y[:clump], ps.z[:clump] = raw
    return with_random_motion(ps, seed)


def run(opts, ps, kick_grid):
    opts.kick_grid = kick_grid
    with TigerPM(opts, ps.n) as t:
        t.set_particles(ps)
        t.chainmesh_create()
        before = t.get_particles()
        t.gravity_long_compute(GRAVITY_LONG_PME)
        g = opts.four_dim
        phi = t.gravity_long_get_phi(Range((0, 0, 0), (g, g, g)))
        t.kick_pme_begin(0, 1.0, 0.01, False)
        t.kick_pme_end()
        t.check_errors()
        return before, phi, t.get_particles(), t.get_forces(), t.chainmesh_offsets()


def test_heavy_cell_queue_matches_grid_and_oracle():
    n = 48
    p = W.accurate_box_params(n)
    # the exact deposit: both launch forms must see the same potential bits
    opts = make_options(n, p["grid"], rs_cells=p["rs_cells"], rcut_over_rs=p["rcut_over_rs"], assign="cloud4",
                        deterministic_deposit=True)
    ps = clumped(n, 40000, 5)
    before, phi, after_q, forces_q, offs = run(opts, ps, 0)
    counts = np.diff(offs)
    heavy = int(np.argmax(counts))
    assert counts[heavy] >= 500 * counts.mean(), (counts[heavy], counts.mean())
    _, _, after_g, forces_g, offs_g = run(opts, ps, 1)
    assert np.array_equal(offs, offs_g)
    for a, b in zip(forces_q + after_q, forces_g + after_g):
        assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))
    C = opts.chain_dim
    sample = np.unique(np.concatenate([[heavy], W.rng(3).choice(C ** 3, 40, replace=False)])).astype(np.int32)
    q = O.Particles(*(np.array(a, copy=True) for a in before))
    kp = kick_params(O, opts, first_call=False, t0=0.01, precision=1)
    ogx, ogy, ogz, opot, cnt, _ = O.kick_pme(kp, q, offs[:-1].copy(), offs[1:].copy(), phi, sink_cells=sample)
    idx = np.concatenate([np.arange(offs[c], offs[c + 1]) for c in sample])
    gx, gy, gz, pot = forces_q
    assert rel_rms(np.stack([gx, gy, gz], 1)[idx], np.stack([ogx, ogy, ogz], 1)[idx]) < 2e-5
    assert rel_rms(pot[idx], opot[idx]) < 2e-5
