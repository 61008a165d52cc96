"""Rung-based kick-drift-kick over one big step (tpm_integrate_*) and the
FP64 diagnostics (tpm_diagnostics).

Each substep is checked against the oracle applied to the device's state
before it: the schedule (largest rung, next tick, drift time, min_rung) is
recomputed exactly; positions after the substep equal the oracle's
fixed-point drift followed by the oracle's restatement of the reference
partition sort, bit for bit; velocities and rungs after the substep's kick
match the oracle's kick (src/kick_pme.cu:319-354) on the same particles and
potential within FP32 tolerance."""
import math

import numpy as np
import pytest

import oracle as O
from helpers import kick_params, rel_rms
from tigerpm_b200 import workloads as W
from tigerpm_b200.api import Range, TigerPM, make_options

pytestmark = pytest.mark.gpu

TICKS = 1 << 31


def _schedule(rung, tick):
    R = int(min(max(int(rung.max()), 0), 31))
    step = 1 << (31 - R)
    t_next = (tick // step + 1) * step
    if t_next >= TICKS:
        return R, t_next, 0
    tz = (t_next & -t_next).bit_length() - 1
    return R, t_next, 31 - tz


def test_integrate_substeps_against_oracle():
    n = 20
    p = W.accurate_box_params(n)
    opts = make_options(n, p["grid"], rs_cells=p["rs_cells"], rcut_over_rs=p["rcut_over_rs"], assign="cloud4")
    ps = W.zeldovich(n, 3, grid=n)
    with TigerPM(opts, ps.n) as t:
        # a big step that spreads the particles over a few rungs
        t.set_particles(ps)
        t.pme_step(0, 1.0, 1.0, True)
        gx, gy, gz, _ = t.get_forces()
        gmed = float(np.median(np.sqrt(gx.astype(np.float64) ** 2 + gy ** 2 + gz ** 2)))
        factor = opts.eta * math.sqrt(opts.hsoft)
        t0 = 6.0 * factor / math.sqrt(gmed)
        t.set_particles(ps)
        t.integrate_begin(t0, 1.0, True)
        tick = 0
        seen_rungs = set()
        for k in range(256):
            x, y, z, vx, vy, vz, r = t.get_particles()
            seen_rungs.update(np.unique(r).tolist())
            R, t_next, min_rung = _schedule(r, tick)
            info = t.integrate_substep()
            assert (info["max_rung"], info["tick"], info["min_rung"]) == (R, t_next, min_rung)
            dt = (t_next - tick) * (t0 / TICKS)
            assert info["drift_dt"] == dt
            # oracle: drift, then the reference partition sort
            q = O.Particles(x.copy(), y.copy(), z.copy(), vx.copy(), vy.copy(), vz.copy(), r.copy())
            O.drift(q, dt)
            pb, pe = O.chainmesh_sort(opts.chain_dim, q)
            x2, y2, z2, vx2, vy2, vz2, r2 = t.get_particles()
            assert np.array_equal(x2, q.x) and np.array_equal(y2, q.y) and np.array_equal(z2, q.z)
            # oracle kick of the due particles on the device's potential
            g = opts.four_dim
            phi = t.gravity_long_get_phi(Range((0, 0, 0), (g, g, g)))
            kp = kick_params(O, opts, min_rung=min_rung, t0=t0, first_call=False, precision=1)
            O.kick_pme(kp, q, pb, pe, phi)
            due = q.rung >= 0  # oracle rungs are updated in place; compare every particle
            V = np.stack([vx2, vy2, vz2], 1).astype(np.float64)
            OV = np.stack([q.vx, q.vy, q.vz], 1).astype(np.float64)
            same = r2 == q.rung
            assert np.mean(~same) < 5e-3
            assert rel_rms(V[same & due], OV[same & due]) < 1e-5
            tick = t_next
            if info["done"]:
                break
        assert tick == TICKS
        assert k >= 2 and len(seen_rungs) >= 2
        # diagnostics: FP64 reductions against numpy on the same arrays
        d = t.diagnostics()
        x, y, z, vx, vy, vz, r = t.get_particles()
        _, _, _, pot = t.get_forces()
        v = np.stack([vx, vy, vz], 1).astype(np.float64)
        assert abs(d["kinetic"] - 0.5 * np.mean(np.sum(v * v, 1))) <= 1e-12 * abs(d["kinetic"]) + 1e-300
        assert abs(d["potential"] - 0.5 * np.mean(pot.astype(np.float64))) <= 1e-12 * abs(d["potential"])
        assert np.allclose(d["momentum"], np.mean(v, 0), rtol=1e-12, atol=1e-18)
        assert d["n"] == ps.n


def test_integrate_errors_and_state():
    opts = make_options(12, 36, rs_cells=2.0, rcut_over_rs=6.0)
    with TigerPM(opts, 12 ** 3) as t:
        t.set_particles(W.uniform(12 ** 3, 4))
        with pytest.raises(Exception):
            t.integrate_substep()  # needs integrate_begin
        with pytest.raises(Exception):
            t.integrate_begin(-1.0)
        t.drift(0.0)
        d = t.diagnostics()
        assert math.isnan(d["potential"]) and d["kinetic"] == 0.0
