"""Generates the golden vectors in tests/golden/ from the reference's own code.

The binaries come from oracle/build_ref.sh, which compiles the reference's
functions from its sources (oracle/_ref/ref_cpu, oracle/_ref/ref_gpu):

  python tests/golden/make_golden.py --cpu          # needs oracle/_ref/ref_cpu
  python tests/golden/make_golden.py --gpu --out D  # needs ref_gpu and a GPU

--cpu writes sort_*.npz (particles_sort + chain-mesh recursion,
src/chainmesh.cpp:168-213), fixed32.npz (tigerpm/fixed.hpp,
tigerpm/gravity_short.hpp:20-22), cloud4.npz (src/gravity_long.cpp:127-138)
and laplacian_*.npz (apply_laplacian, src/gravity_long.cpp:201-245).
--gpu writes kick_*.npz (kick_pme + kick_pme_kernel, src/kick_pme.cu:128-621)
and ewald_*.npz (gravity_short_ewald_call_kernel, src/gravity_short.cu).

Every input is drawn from a seeded generator, so a rerun reproduces the files.
Inputs to the reference's GPU code are checked on the host first: positions
below 2^32 - 4096 (so the reference's 6-point stencil, which reads up to
int(x*N) + 3, stays inside its padded potential box), rungs that the oracle
keeps below 20, and a cell table that covers every particle once.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from oracle import ref_runner as R  # noqa: E402

U32_MAX_SAFE = (1 << 32) - 4096


def _u32(g, n, hi=1 << 32):
    return g.integers(0, hi, n, dtype=np.uint64).astype(np.uint32)


def _motion(g, n, max_rung):
    v = [g.normal(0, 1e-3, n).astype(np.float32) for _ in range(3)]
    r = g.integers(0, max_rung + 1, n).astype(np.int8)
    return v, r


def sort_inputs():
    """(name, C, x, y, z) cases: uniform, clustered, duplicates, positions on
    and next to every cell threshold, single cell, empty."""
    g = np.random.default_rng(20211)
    cases = []
    for C, n in ((6, 3000), (7, 2500), (8, 4096), (12, 5000)):
        cases.append((f"uniform_C{C}", C, _u32(g, n), _u32(g, n), _u32(g, n)))
    # clustered: three Gaussian blobs, periodic wrap
    n = 4000
    ctr = g.random((3, 3))
    lab = g.integers(0, 3, n)
    pos = (ctr[lab] + g.normal(0, 0.03, (n, 3))) % 1.0
    raw = np.minimum((pos * 4294967296.0).astype(np.uint64), (1 << 32) - 1).astype(np.uint32)
    cases.append(("clustered_C9", 9, raw[:, 0].copy(), raw[:, 1].copy(), raw[:, 2].copy()))
    # thresholds: fixed32(k/C) - 1, +0, +1 for every boundary k, in all dims
    for C in (5, 6, 10):
        t = []
        for k in range(C + 1):
            b = O.fixed32_from_double(k / C)
            for d in (-1, 0, 1):
                v = b + d
                if 0 <= v < (1 << 32):
                    t.append(v)
        t = np.array(sorted(set(t)), np.uint64)
        m = 1500
        cases.append((f"thresholds_C{C}", C, t[g.integers(0, t.size, m)].astype(np.uint32),
                      t[g.integers(0, t.size, m)].astype(np.uint32),
                      t[g.integers(0, t.size, m)].astype(np.uint32)))
    # many exact duplicates
    base = _u32(g, 40)
    idx = g.integers(0, 40, 1200)
    cases.append(("duplicates_C4", 4, base[idx], base[(idx + 7) % 40], base[(idx * 3) % 40]))
    # everything in one cell, and C = 1, and n = 0, 1
    cases.append(("one_cell_C5", 5, _u32(g, 700, 1 << 28), _u32(g, 700, 1 << 28), _u32(g, 700, 1 << 28)))
    cases.append(("single_C1", 1, _u32(g, 33), _u32(g, 33), _u32(g, 33)))
    cases.append(("empty_C3", 3, np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.uint32)))
    cases.append(("one_C4", 4, _u32(g, 1), _u32(g, 1), _u32(g, 1)))
    return cases


def make_cpu(out):
    g = np.random.default_rng(7)
    for name, C, x, y, z in sort_inputs():
        n = x.size
        (vx, vy, vz), rung = _motion(g, n, 5)
        (sx, sy, sz, svx, svy, svz, sr), cells = R.sort(C, x, y, z, vx, vy, vz, rung)
        assert (cells >= 0).all(), name
        np.savez_compressed(os.path.join(out, f"sort_{name}.npz"), C=np.int32(C), x=x, y=y, z=z,
                            vx=vx, vy=vy, vz=vz, rung=rung, out_x=sx, out_y=sy, out_z=sz,
                            out_vx=svx, out_vy=svy, out_vz=svz, out_rung=sr, pbegin=cells[:, 0].copy(),
                            pend=cells[:, 1].copy())
    # fixed32: conversions and the periodic distance
    m = 4000
    xs = np.concatenate([g.random(m), np.array([0.0, 0.5, 0.25, 1 / 3, 2 / 3, 1 / 7, 0.1, 0.9,
                                                0.999999999, 1e-10, 2.0 ** -32, 1 - 2.0 ** -33])])
    xs = np.concatenate([xs, np.arange(1, 64) / 64.0, np.arange(1, 97) / 97.0])
    a = _u32(g, xs.size)
    b = _u32(g, xs.size)
    b[:8] = a[:8]
    b[8:16] = a[8:16] + np.uint32(1 << 31)
    raw, tf, td, dist = R.fixed(xs, a, b)
    np.savez_compressed(os.path.join(out, "fixed32.npz"), x=xs, a=a, b=b, raw=raw, to_float=tf,
                        to_double=td, distance=dist)
    # cloud4 over its support and beyond
    xc = np.concatenate([np.linspace(-2.5, 2.5, 5001), g.uniform(-3, 3, 2000), [-2.0, -1.0, 0.0, 1.0, 2.0]])
    np.savez_compressed(os.path.join(out, "cloud4.npz"), x=xc, w=R.cloud4(xc))
    # apply_laplacian on a random half-spectrum, PM (0) and PME (1)
    for N, rs_cells in ((8, 1.0), (12, 1.25), (16, 2.0)):
        shape = (N, N, N // 2 + 1)
        Y = (g.standard_normal(shape) + 1j * g.standard_normal(shape)).astype(np.complex64)
        res = {}
        for typ in (0, 1):
            res[f"out{typ}"] = R.laplacian(N, rs_cells, typ, Y)
        np.savez_compressed(os.path.join(out, f"laplacian_N{N}.npz"), N=np.int32(N),
                            rs_cells=np.float64(rs_cells), Y=Y, **res)
    # initial conditions: the reference's power-table reader, log-cubic
    # interpolation, sigma8 normalisation and growth factor, run on a table of
    # our own (P ~ k T(k)^2 with the BBKS transfer function, Bardeen et al.
    # 1986, Gamma = 0.21), written in power.init's format
    tk = np.logspace(-4, 2, 300)
    q = tk / 0.21
    T = np.log1p(2.34 * q) / (2.34 * q) * (1 + 3.89 * q + (16.1 * q) ** 2 + (5.46 * q) ** 3 + (6.71 * q) ** 4) ** -0.25
    tp = 2.0e4 * tk * T ** 2
    tk = np.array([float(f"{v:.5E}") for v in tk])
    tp = np.array([float(f"{v:.5E}") for v in tp])
    hubble, sigma8 = 0.7, 0.84
    ks = np.concatenate([np.logspace(-4.6, 2.3, 400) * hubble, 2 * np.pi / 100.0 * np.sqrt(np.arange(1, 200))])
    oa = np.array([[0.3, 1 / 3], [0.3, 0.5], [0.3, 1.0], [0.25, 0.1], [1.0, 0.5], [0.3, 1 / 1.5]])
    pk, gf = R.power(tk, tp, hubble, sigma8, ks, oa)
    np.savez_compressed(os.path.join(out, "ic_power.npz"), table_k=tk, table_p=tp, hubble=np.float64(hubble),
                        sigma8=np.float64(sigma8), k=ks, P=pk, omega_a=oa, growth=gf)


def kick_inputs():
    """Kick cases: (name, C, four_o_chain, rs_cells, hsoft, GM, eta, min_rung,
    t0, scale, first_call, positions kind, n)."""
    return [
        ("uniform_first", 6, 4, 1.25, 0.004, 1.0 / 3000, 0.2, 0, 1.0, 1.0, 1, "uniform", 3000),
        ("clustered_rungs", 5, 4, 1.5, 0.003, 1.0 / 4000, 0.2, 1, 0.5, 0.8, 0, "clustered", 4000),
        ("sparse_C3", 3, 4, 1.0, 0.01, 1.0 / 60, 0.3, 0, 1.0, 1.0, 0, "uniform", 60),
    ]


def kick_case(name, C, foc, rs_cells, hsoft, GM, eta, min_rung, t0, scale, first_call, kind, n, seed):
    g = np.random.default_rng(seed)
    if kind == "uniform":
        x, y, z = (_u32(g, n, U32_MAX_SAFE) for _ in range(3))
    else:
        ctr = g.random((4, 3)) * 0.8 + 0.1
        lab = g.integers(0, 4, n)
        pos = (ctr[lab] + g.normal(0, 0.04, (n, 3))) % 1.0
        raw = np.minimum((pos * 4294967296.0).astype(np.uint64), U32_MAX_SAFE - 1).astype(np.uint32)
        x, y, z = raw[:, 0].copy(), raw[:, 1].copy(), raw[:, 2].copy()
    (vx, vy, vz), rung = _motion(g, n, 4)
    (sx, sy, sz, svx, svy, svz, sr), cells = R.sort(C, x, y, z, vx, vy, vz, rung)
    assert (cells >= 0).all() and cells[-1, 1] == n
    assert np.array_equal(np.sort(np.concatenate([np.arange(a, b) for a, b in cells])), np.arange(n))
    assert int(max(sx.max(), sy.max(), sz.max())) < U32_MAX_SAFE
    N = foc * C
    rs = rs_cells / N
    phi = O.gravity_long(N, rs_cells, 0, sx, sy, sz, pme=1).astype(np.float32)
    # host check of the rungs the reference will assign (oracle, FP32 arithmetic)
    p = O.Particles(sx.copy(), sy.copy(), sz.copy(), svx.copy(), svy.copy(), svz.copy(), sr.copy())
    kp = O.KickParams(N=N, C=C, rs=rs, GM=GM, eta=eta, hsoft=hsoft, rcut=0.0, min_rung=min_rung,
                      scale=scale, t0=t0, first_call=first_call, precision=0)
    O.kick_pme(kp, p, cells[:, 0].copy(), cells[:, 1].copy(), phi)
    assert int(p.rung.max()) < 20, int(p.rung.max())
    res = R.kick(C, N, foc, rs, GM, eta, hsoft, min_rung, scale, t0, first_call,
                 (sx, sy, sz, svx, svy, svz, sr), cells, phi)
    return dict(C=np.int32(C), N=np.int32(N), four_o_chain=np.int32(foc), rs=np.float64(rs),
                rs_cells=np.float64(rs_cells), hsoft=np.float64(hsoft), GM=np.float64(GM),
                eta=np.float64(eta), min_rung=np.int32(min_rung), t0=np.float64(t0),
                scale=np.float64(scale), first_call=np.int32(first_call), x=sx, y=sy, z=sz, vx=svx,
                vy=svy, vz=svz, rung=sr, pbegin=cells[:, 0].copy(), pend=cells[:, 1].copy(), phi=phi,
                out_vx=res["vx"], out_vy=res["vy"], out_vz=res["vz"], out_rung=res["rung"],
                out_gx=res["gx"], out_gy=res["gy"], out_gz=res["gz"], out_pot=res["pot"])


def make_gpu(out):
    for i, case in enumerate(kick_inputs()):
        d = kick_case(*case, seed=300 + i)
        np.savez_compressed(os.path.join(out, f"kick_{case[0]}.npz"), **d)
    for name, n, ns, hsoft, seed in (("uniform", 3000, 48, 0.004, 11), ("clustered", 2000, 32, 0.002, 12)):
        g = np.random.default_rng(seed)
        if name == "uniform":
            x, y, z = (_u32(g, n) for _ in range(3))
        else:
            ctr = g.random((2, 3))
            lab = g.integers(0, 2, n)
            pos = (ctr[lab] + g.normal(0, 0.05, (n, 3))) % 1.0
            raw = np.minimum((pos * 4294967296.0).astype(np.uint64), (1 << 32) - 1).astype(np.uint32)
            x, y, z = raw[:, 0].copy(), raw[:, 1].copy(), raw[:, 2].copy()
        sel = g.choice(n, ns, replace=False)
        sx, sy, sz = x[sel], y[sel], z[sel]
        phi, gx, gy, gz = R.ewald(x, y, z, sx, sy, sz, hsoft)
        np.savez_compressed(os.path.join(out, f"ewald_{name}.npz"), x=x, y=y, z=z, sink_index=sel.astype(np.int64),
                            hsoft=np.float64(hsoft), phi=phi, gx=gx, gy=gy, gz=gz)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cpu", action="store_true")
    ap.add_argument("--gpu", action="store_true")
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if a.cpu:
        make_cpu(a.out)
    if a.gpu:
        make_gpu(a.out)


if __name__ == "__main__":
    main()
