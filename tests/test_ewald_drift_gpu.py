"""FP64 Ewald on the device vs the oracle's FP64 restatement of
gravity_ewald_kernel (src/gravity_short.cu:93-201), and the fixed-point
drift bit-exact vs the oracle."""
import numpy as np
import pytest

import oracle as O
from helpers import oracle_particles, particle_set, rel_rms, with_random_motion
from tigerpm_b200 import workloads as W
from tigerpm_b200.api import TigerPM, make_options

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["uniform", "halos"])
def test_ewald_methods_match_oracle(kind):
    ps = particle_set(kind, 16, 13)
    opts = make_options(16, 16, rs_cells=1.0)
    idx = W.sample_indices(ps.n, 24, 5)
    sx, sy, sz = ps.x[idx], ps.y[idx], ps.z[idx]
    sx[0] = sx[0] + 1000  # a near pair that is not the sink itself
    with TigerPM(opts, ps.n) as t:
        t.set_particles(ps)
        p0, g0 = t.gravity_short_ewald_call_kernel(sx, sy, sz, method=0)
        p1, g1 = t.gravity_short_ewald_call_kernel(sx, sy, sz, method=1)
    op, ogx, ogy, ogz = O.ewald_ref(ps.x, ps.y, ps.z, sx, sy, sz, opts.hsoft)
    OG = np.stack([ogx, ogy, ogz], 1)
    assert rel_rms(np.stack(g0, 1), OG) < 1e-12
    assert rel_rms(p0, op) < 1e-12
    assert rel_rms(np.stack(g1, 1), OG) < 1e-9
    assert rel_rms(p1, op) < 1e-9


def test_drift_bit_exact():
    ps = with_random_motion(particle_set("uniform", 20, 17), 17, vscale=0.3)
    ps.vx[:5] = [0.0, -0.0, 1e-12, -3.7e-9, 0.49999]
    opts = make_options(20, 16, rs_cells=1.0)
    for dt in (1e-3, 0.37, 1.0 / 3.0):
        with TigerPM(opts, ps.n) as t:
            t.set_particles(ps)
            t.drift(dt)
            x, y, z, *_ = t.get_particles()
        p = oracle_particles(O, ps)
        O.drift(p, dt)
        assert np.array_equal(x, p.x) and np.array_equal(y, p.y) and np.array_equal(z, p.z)


def test_drift_rejects_huge_step():
    ps = particle_set("uniform", 8, 1)
    ps.vx[:] = 1e9
    opts = make_options(8, 8, rs_cells=1.0)
    with TigerPM(opts, ps.n) as t:
        t.set_particles(ps)
        with pytest.raises(Exception):
            t.drift(10.0)
