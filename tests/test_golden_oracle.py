"""Pins the oracle to the reference: its restatements against golden vectors
recorded from the reference's own functions, compiled from the reference's
sources (oracle/build_ref.sh) and run by tests/golden/make_golden.py.

  sort_*      particles_sort + chain-mesh recursion (src/chainmesh.cpp:168-213,
              src/particles.cpp:414-444): bit-exact
  fixed32     fixed32(double), to_float, to_double, distance (tigerpm/fixed.hpp,
              tigerpm/gravity_short.hpp:20-22): bit-exact
  cloud4      src/gravity_long.cpp:127-138: bit-exact (same FP64 expression)
  laplacian_* apply_laplacian (src/gravity_long.cpp:201-245) on complex<float>:
              the oracle works in FP64, so within FP32 rounding (2e-6 relative)
  kick_*      kick_pme_kernel on a B200 (src/kick_pme.cu:128-357), given the
              same sorted particles, cell table and potential: the oracle's
              FP32 path within 5e-6 relative RMS (measured 2e-7..5e-7: libm vs
              CUDA's sqrt/rsqrt and summation order), rungs identical but for
              power-of-two ties
  ewald_*     gravity_ewald_kernel on a B200 (src/gravity_short.cu:93-201):
              the oracle's restatement within 1e-5 relative RMS (measured
              1e-7 on forces, 2e-6 on the uniform case's potential, where
              the sum cancels)
"""
import numpy as np
import pytest

import oracle as O
from golden_io import load, names
from helpers import rel_rms


@pytest.mark.parametrize("case", names("sort"))
def test_sort_bit_exact(case):
    d = load("sort_" + case)
    C = int(d["C"])
    p = O.Particles(*(d[k].copy() for k in ("x", "y", "z", "vx", "vy", "vz", "rung")))
    pb, pe = O.chainmesh_sort(C, p)
    for k, a in zip(("x", "y", "z"), (p.x, p.y, p.z)):
        assert np.array_equal(a, d["out_" + k]), k
    for k, a in zip(("vx", "vy", "vz"), (p.vx, p.vy, p.vz)):
        assert np.array_equal(a.view(np.uint32), d["out_" + k].view(np.uint32)), k
    assert np.array_equal(p.rung, d["out_rung"])
    assert np.array_equal(pb, d["pbegin"]) and np.array_equal(pe, d["pend"])


def test_fixed32_bit_exact():
    d = load("fixed32")
    assert np.array_equal(O.fixed32_from_double_array(d["x"]), d["raw"])
    tf, td, ds = O.fixed32_convert_array(d["a"], d["b"])
    assert np.array_equal(tf.view(np.uint32), d["to_float"].view(np.uint32))
    assert np.array_equal(td.view(np.uint64), d["to_double"].view(np.uint64))
    assert np.array_equal(ds.view(np.uint32), d["distance"].view(np.uint32))


def test_cloud4_bit_exact():
    d = load("cloud4")
    assert np.array_equal(O.cloud4(d["x"]).view(np.uint64), d["w"].view(np.uint64))


@pytest.mark.parametrize("case", names("laplacian"))
@pytest.mark.parametrize("typ", [0, 1])
def test_laplacian(case, typ):
    d = load("laplacian_" + case)
    ref = d[f"out{typ}"].astype(np.complex128)
    mine = O.green_apply(d["Y"], float(d["rs_cells"]), pme=typ, deconv_order=4)
    scale = np.abs(ref).max()
    assert np.abs(mine - ref).max() <= 2e-6 * scale
    assert np.all(mine.ravel()[0] == 0) and np.all(ref.ravel()[0] == 0)


@pytest.mark.parametrize("case", names("kick"))
def test_kick(case):
    d = load("kick_" + case)
    N, C = int(d["N"]), int(d["C"])
    p = O.Particles(*(d[k].copy() for k in ("x", "y", "z", "vx", "vy", "vz", "rung")))
    kp = O.KickParams(N=N, C=C, rs=float(d["rs"]), GM=float(d["GM"]), eta=float(d["eta"]),
                      hsoft=float(d["hsoft"]), rcut=0.0, min_rung=int(d["min_rung"]),
                      scale=float(d["scale"]), t0=float(d["t0"]), first_call=int(d["first_call"]),
                      precision=0)
    gx, gy, gz, pot, counts, bad = O.kick_pme(kp, p, d["pbegin"].copy(), d["pend"].copy(), d["phi"])
    active = d["rung"] >= int(d["min_rung"])
    assert active.any()
    G = np.stack([gx, gy, gz], 1)[active]
    RG = np.stack([d["out_gx"], d["out_gy"], d["out_gz"]], 1)[active]
    assert rel_rms(G, RG) < 5e-6
    assert rel_rms(pot[active], d["out_pot"][active]) < 5e-6
    assert np.mean(p.rung != d["out_rung"]) < 2e-3
    assert np.abs(p.rung.astype(int) - d["out_rung"].astype(int)).max() <= 1
    # inactive sinks are untouched by both
    assert np.array_equal(p.rung[~active], d["out_rung"][~active])
    same = p.rung == d["out_rung"]
    V = np.stack([p.vx, p.vy, p.vz], 1)[same]
    RV = np.stack([d["out_vx"], d["out_vy"], d["out_vz"]], 1)[same]
    assert rel_rms(V, RV) < 2e-5


@pytest.mark.parametrize("case", names("ewald"))
def test_ewald(case):
    d = load("ewald_" + case)
    s = d["sink_index"]
    x, y, z = d["x"], d["y"], d["z"]
    phi, gx, gy, gz = O.ewald_ref(x, y, z, x[s].copy(), y[s].copy(), z[s].copy(), float(d["hsoft"]))
    assert rel_rms(np.stack([gx, gy, gz], 1), np.stack([d["gx"], d["gy"], d["gz"]], 1)) < 1e-5
    assert rel_rms(phi, d["phi"]) < 1e-5
