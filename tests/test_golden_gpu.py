"""Device path against golden vectors recorded from the reference's own code
(tests/golden/make_golden.py; inputs and outputs of the reference's
chain-mesh sort, kick_pme and Ewald kernels, compiled from its sources).

  sort_*   device parity sort: bit-exact permutation and cell table
  kick_*   (a) the golden potential loaded with gravity_long_set_phi, then
           the device kick: forces and potentials within 2e-5 relative RMS of
           the reference kernel (FP32 arithmetic on both sides; erfc/exp/rsqrt
           and summation order differ), rungs equal but for power-of-two ties;
           (b) the whole device path (sort -> gravity_long -> kick): device
           FP32 potential within 1e-5 of the golden FP64-built one, forces
           within 5e-5
  ewald_*  tpm_gravity_short_ewald method 0 (the reference's sum) and method
           1 (alpha = 6, FP64) against the reference kernel (FP32 terms
           accumulated in FP64) within 1e-5; the no-alloc entry point is
           checked against the same vectors in test_zz_no_alloc.py
"""
import numpy as np
import pytest

from golden_io import load, names
from helpers import rel_rms
from tigerpm_b200 import workloads as W
from tigerpm_b200.api import GRAVITY_LONG_PME, TigerPM, TPMError, make_options

pytestmark = pytest.mark.gpu


def _ps(d, prefix=""):
    return W.ParticleSet(*(d[prefix + k].copy() for k in ("x", "y", "z", "vx", "vy", "vz", "rung")))


@pytest.mark.parametrize("case", names("sort"))
def test_sort_golden(case):
    d = load("sort_" + case)
    C = int(d["C"])
    ps = _ps(d)
    opts = make_options(16, 16, chain=C, sort="parity")
    if C < 3:
        # the device needs 27 distinct neighbour cells; the reference recursion accepts any C
        with pytest.raises(TPMError):
            TigerPM(opts, max(ps.n, 1))
        return
    with TigerPM(opts, max(ps.n, 1)) as t:
        t.set_particles(ps)
        t.chainmesh_create()
        x, y, z, vx, vy, vz, r = t.get_particles()
        offs = t.chainmesh_offsets()
    for k, a in zip(("x", "y", "z"), (x, y, z)):
        assert np.array_equal(a, d["out_" + k]), k
    for k, a in zip(("vx", "vy", "vz"), (vx, vy, vz)):
        assert np.array_equal(a.view(np.uint32), d["out_" + k].view(np.uint32)), k
    assert np.array_equal(r, d["out_rung"])
    assert np.array_equal(offs[:-1], d["pbegin"]) and np.array_equal(offs[1:], d["pend"])


def _kick_opts(d):
    o = make_options(16, int(d["N"]), chain=int(d["C"]), rs_cells=float(d["rs_cells"]), rcut_over_rs=0.0,
                     assign="cloud4", GM=float(d["GM"]))
    o.hsoft = float(d["hsoft"])
    o.eta = float(d["eta"])
    return o


def _check_kick(d, after, forces, tol_g):
    gx, gy, gz, pot = forces
    active = d["rung"] >= int(d["min_rung"])
    G = np.stack([gx, gy, gz], 1)[active]
    RG = np.stack([d["out_gx"], d["out_gy"], d["out_gz"]], 1)[active]
    assert rel_rms(G, RG) < tol_g, rel_rms(G, RG)
    assert rel_rms(pot[active], d["out_pot"][active]) < tol_g
    r = after[6]
    assert np.mean(r != d["out_rung"]) < 2e-3
    assert np.abs(r.astype(int) - d["out_rung"].astype(int)).max() <= 1
    assert np.array_equal(r[~active], d["out_rung"][~active])
    for k, a in zip(("vx", "vy", "vz"), after[3:6]):
        assert np.array_equal(a[~active].view(np.uint32), d[k][~active].view(np.uint32))
    same = r == d["out_rung"]
    V = np.stack(after[3:6], 1)[same]
    RV = np.stack([d["out_vx"], d["out_vy"], d["out_vz"]], 1)[same]
    assert rel_rms(V, RV) < tol_g


@pytest.mark.parametrize("case", names("kick"))
def test_kick_golden_given_phi(case):
    d = load("kick_" + case)
    with TigerPM(_kick_opts(d), d["x"].size) as t:
        t.set_particles(_ps(d))
        t.chainmesh_create()
        offs = t.chainmesh_offsets()
        # an already partitioned set keeps its order under the reference's partition
        assert np.array_equal(offs[:-1], d["pbegin"]) and np.array_equal(offs[1:], d["pend"])
        t.gravity_long_set_phi(d["phi"])
        t.kick_pme_begin(int(d["min_rung"]), float(d["scale"]), float(d["t0"]), bool(d["first_call"]))
        t.kick_pme_end()
        after = t.get_particles()
        forces = t.get_forces()
    assert np.array_equal(after[0], d["x"])
    _check_kick(d, after, forces, 2e-5)


@pytest.mark.parametrize("case", names("kick"))
def test_kick_golden_whole_path(case):
    d = load("kick_" + case)
    N = int(d["N"])
    with TigerPM(_kick_opts(d), d["x"].size) as t:
        t.set_particles(_ps(d))
        t.chainmesh_create()
        t.gravity_long_compute(GRAVITY_LONG_PME)
        from tigerpm_b200.api import Range
        phi = t.gravity_long_get_phi(Range((0, 0, 0), (N, N, N)))
        t.kick_pme_begin(int(d["min_rung"]), float(d["scale"]), float(d["t0"]), bool(d["first_call"]))
        t.kick_pme_end()
        after = t.get_particles()
        forces = t.get_forces()
    assert rel_rms(phi.ravel(), d["phi"].ravel()) < 1e-5
    _check_kick(d, after, forces, 5e-5)


@pytest.mark.parametrize("case", names("ewald"))
@pytest.mark.parametrize("method", [0, 1])
def test_ewald_golden(case, method):
    d = load("ewald_" + case)
    x, y, z = d["x"], d["y"], d["z"]
    s = d["sink_index"]
    n = x.size
    o = make_options(16, 16, chain=4)
    o.hsoft = float(d["hsoft"])
    ps = W.ParticleSet(x.copy(), y.copy(), z.copy(), np.zeros(n, np.float32), np.zeros(n, np.float32),
                       np.zeros(n, np.float32), np.zeros(n, np.int8))
    with TigerPM(o, n) as t:
        t.set_particles(ps)
        phi, g = t.gravity_short_ewald_call_kernel(x[s], y[s], z[s], method=method)
    assert rel_rms(np.stack(g, 1), np.stack([d["gx"], d["gy"], d["gz"]], 1)) < 1e-5
    assert rel_rms(phi, d["phi"]) < 1e-5

