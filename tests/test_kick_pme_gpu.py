"""Device kick (interpolation + PP + rung kick) vs the oracle's restatement
of kick_pme_kernel (src/kick_pme.cu:128-357), on the same sorted particles
and the same potential; and the whole kick vs the FP64 Ewald sum."""
import math

import numpy as np
import pytest

import oracle as O
from helpers import kick_params, oracle_particles, particle_set, rel_rms, with_random_motion
from tigerpm_b200 import workloads as W
from tigerpm_b200.api import GRAVITY_LONG_PME, Range, TigerPM, make_options

pytestmark = pytest.mark.gpu


def device_kick(ps, opts, min_rung=0, first_call=True, t0=1.0, scale=1.0):
    with TigerPM(opts, ps.n) as t:
        t.set_particles(ps)
        t.chainmesh_create()
        sorted_ps = t.get_particles()
        t.gravity_long_compute(GRAVITY_LONG_PME)
        g = opts.four_dim
        phi = t.gravity_long_get_phi(Range((0, 0, 0), (g, g, g)))
        t.kick_pme_begin(min_rung, scale, t0, first_call)
        t.kick_pme_end()
        after = t.get_particles()
        forces = t.get_forces()
        pb = t.chainmesh_offsets()
    return sorted_ps, phi, after, forces, pb


CASES = [
    # kind, n_side, grid, rs_cells, rcut_over_rs, assign
    ("uniform", 20, 20, 1.0, 0.0, "cloud4"),     # the reference scheme: no cutoff
    ("uniform", 24, 32, 1.25, 4.5, "cic"),
    ("zeldovich", 24, 48, 2.0, 5.5, "tsc"),
    ("halos", 24, 24, 1.25, 4.5, "cloud4"),
]


@pytest.mark.parametrize("kind,n_side,grid,rs,rcut,assign", CASES)
def test_kick_matches_oracle(kind, n_side, grid, rs, rcut, assign):
    ps = with_random_motion(particle_set(kind, n_side, 21, grid), 21)
    opts = make_options(n_side, grid, rs_cells=rs, rcut_over_rs=rcut, assign=assign)
    (x, y, z, vx, vy, vz, r), phi, after, (gx, gy, gz, pot), offs = device_kick(ps, opts, first_call=False, t0=0.01)
    p = O.Particles(x.copy(), y.copy(), z.copy(), vx.copy(), vy.copy(), vz.copy(), r.copy())
    kp = kick_params(O, opts, first_call=False, t0=0.01, precision=1)
    ogx, ogy, ogz, opot, counts, bad = O.kick_pme(kp, p, offs[:-1].copy(), offs[1:].copy(), phi)
    G = np.stack([gx, gy, gz], 1)
    OG = np.stack([ogx, ogy, ogz], 1)
    err_g = rel_rms(G, OG)
    err_p = rel_rms(pot, opot)
    assert err_g < 1e-5, err_g
    assert err_p < 1e-5, err_p
    # rungs: identical except where the FP32 force sits on a power-of-two boundary
    assert np.mean(after[6] != p.rung) < 1e-3
    same = after[6] == p.rung
    V = np.stack(after[3:6], 1)[same]
    OV = np.stack([p.vx, p.vy, p.vz], 1)[same]
    assert rel_rms(V, OV) < 1e-5


def test_reference_fp32_arithmetic_close():
    """The oracle's FP32 path follows the reference's arithmetic (float
    to_float positions, A&S erfc, sequential sums); the device agrees with it
    to FP32 rounding."""
    ps = particle_set("uniform", 20, 5)
    opts = make_options(20, 20, rs_cells=1.0)
    (x, y, z, vx, vy, vz, r), phi, after, (gx, gy, gz, pot), offs = device_kick(ps, opts)
    p = O.Particles(x.copy(), y.copy(), z.copy(), vx.copy(), vy.copy(), vz.copy(), r.copy())
    kp = kick_params(O, opts, precision=0)
    ogx, ogy, ogz, opot, counts, bad = O.kick_pme(kp, p, offs[:-1].copy(), offs[1:].copy(), phi)
    assert rel_rms(np.stack([gx, gy, gz], 1), np.stack([ogx, ogy, ogz], 1)) < 5e-5
    assert rel_rms(pot, opot) < 5e-5


def test_min_rung_only_kicks_active():
    ps = with_random_motion(particle_set("uniform", 16, 3), 3, max_rung=4)
    opts = make_options(16, 16, rs_cells=1.0)
    (x, y, z, vx, vy, vz, r), phi, after, (gx, gy, gz, pot), offs = device_kick(ps, opts, min_rung=2,
                                                                                first_call=False, t0=0.01)
    inactive = r < 2
    assert np.array_equal(after[3][inactive], vx[inactive])
    assert np.array_equal(after[6][inactive], r[inactive])
    assert np.all(gx[inactive] == 0)
    assert np.all(gx[~inactive] != 0)


def test_kick_vs_ewald_small():
    """Whole kick vs the FP64 Ewald sum (reference structure, alpha = 2) on
    sampled particles: the error of the accurate form is below 1e-4."""
    ps = particle_set("uniform", 24, 31)
    opts = make_options(24, 48, rs_cells=2.0, rcut_over_rs=5.5, assign="cloud4")
    with TigerPM(opts, ps.n) as t:
        t.set_particles(ps)
        t.chainmesh_create()
        t.gravity_long_compute(GRAVITY_LONG_PME)
        t.kick_pme_begin(0, 1.0, 1.0, True)
        e0 = t.gravity_short_ewald_compare(48, seed=2, method=0)
        e1 = t.gravity_short_ewald_compare(48, seed=2, method=1)
    assert e0["force_rms_vector"] < 1.5e-4, e0
    assert abs(e0["force_rms_vector"] - e1["force_rms_vector"]) < 1e-7
