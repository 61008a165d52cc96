"""Drives the reference binaries built by oracle/build_ref.sh (oracle/_ref/).

TEST INFRASTRUCTURE ONLY: used by tests/golden/make_golden.py to record what
the reference's own code computes; the product never calls it.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "_ref")


def _run(exe, args, payload: bytes) -> bytes:
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            f.write(payload)
        subprocess.run([os.path.join(REF, exe)] + [str(a) for a in args if a is not None] + [fin, fout], check=True,
                       stdout=subprocess.DEVNULL)
        with open(fout, "rb") as f:
            return f.read()


def sort(C: int, x, y, z, vx, vy, vz, rung):
    """particles_sort + chain-mesh recursion (src/chainmesh.cpp:168-213)."""
    n = x.size
    pay = struct.pack("<q", n) + b"".join(np.ascontiguousarray(a).tobytes() for a in (x, y, z, vx, vy, vz, rung))
    out = _run("ref_cpu", ["sort", C, None, None], pay)
    o = 0
    res = []
    for dt in ("<u4",) * 3 + ("<f4",) * 3:
        res.append(np.frombuffer(out, dt, n, o).copy())
        o += 4 * n
    res.append(np.frombuffer(out, "i1", n, o).copy())
    o += n
    cells = np.frombuffer(out, "<i4", 2 * C ** 3, o).reshape(-1, 2).copy()
    return res, cells


def cloud4(x):
    x = np.ascontiguousarray(x, np.float64)
    out = _run("ref_cpu", ["cloud4", None, None], struct.pack("<q", x.size) + x.tobytes())
    return np.frombuffer(out, "<f8").copy()


def laplacian(N: int, rs_cells: float, typ: int, Y):
    Y = np.ascontiguousarray(Y, np.complex64)
    out = _run("ref_cpu", ["laplacian", N, repr(rs_cells), typ, None, None], Y.tobytes())
    return np.frombuffer(out, np.complex64).reshape(Y.shape).copy()


def fixed(x, a, b):
    m = x.size
    pay = struct.pack("<q", m) + np.ascontiguousarray(x, np.float64).tobytes() + \
        np.ascontiguousarray(a, np.uint32).tobytes() + np.ascontiguousarray(b, np.uint32).tobytes()
    out = _run("ref_cpu", ["fixed", None, None], pay)
    raw = np.frombuffer(out, "<u4", m, 0).copy()
    tf = np.frombuffer(out, "<f4", m, 4 * m).copy()
    td = np.frombuffer(out, "<f8", m, 8 * m).copy()
    dist = np.frombuffer(out, "<f4", m, 16 * m).copy()
    return raw, tf, td, dist


def kick(C, N, four_o_chain, rs, GM, eta, hsoft, min_rung, scale, t0, first_call, arrays, cells, phi):
    """The reference's kick_pme on the GPU (src/kick_pme.cu:390-621)."""
    x, y, z, vx, vy, vz, rung = arrays
    n = x.size
    pay = struct.pack("<qiiiddddiddi", n, C, N, four_o_chain, rs, GM, eta, hsoft, min_rung, scale, t0, first_call)
    pay += b"".join(np.ascontiguousarray(a).tobytes() for a in (x, y, z, vx, vy, vz, rung))
    pay += np.ascontiguousarray(cells, np.int32).tobytes() + np.ascontiguousarray(phi, np.float32).tobytes()
    out = _run("ref_gpu", ["kick", None, None], pay)
    o = 0
    res = {}
    for k in ("vx", "vy", "vz"):
        res[k] = np.frombuffer(out, "<f4", n, o).copy()
        o += 4 * n
    res["rung"] = np.frombuffer(out, "i1", n, o).copy()
    o += n
    for k in ("gx", "gy", "gz", "pot"):
        res[k] = np.frombuffer(out, "<f4", n, o).copy()
        o += 4 * n
    return res


def ewald(x, y, z, sx, sy, sz, hsoft):
    """gravity_short_ewald_call_kernel on the GPU (src/gravity_short.cu:10-91)."""
    n, ns = x.size, sx.size
    pay = struct.pack("<qqd", n, ns, hsoft) + b"".join(np.ascontiguousarray(a, np.uint32).tobytes()
                                                       for a in (x, y, z, sx, sy, sz))
    out = _run("ref_gpu", ["ewald", None, None], pay)
    v = np.frombuffer(out, "<f8").reshape(4, ns).copy()
    return v[0], v[1], v[2], v[3]


def power(table_k, table_p, hubble: float, sigma8: float, k, omega_a):
    """read_power_spectrum + power_spectrum_function + growth_factor
    (src/initialize.cpp:10-83,182-211) on a power.init written from the
    given table (k in h/Mpc, P in (Mpc/h)^3).  Returns (P(k), growth)."""
    k = np.ascontiguousarray(k, np.float64)
    oa = np.ascontiguousarray(omega_a, np.float64).reshape(-1, 2)
    pay = (struct.pack("<q", k.size) + k.tobytes() + struct.pack("<q", oa.shape[0]) + oa.tobytes())
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "power.init"), "w") as f:
            for a, b in zip(table_k, table_p):
                f.write(f"   {a:.5E}   {b:.5E}\n")
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            f.write(pay)
        subprocess.run([os.path.join(REF, "ref_cpu"), "power", repr(hubble), repr(sigma8), fin, fout], check=True,
                       stdout=subprocess.DEVNULL, cwd=d)
        out = np.fromfile(fout, np.float64)
    return out[:k.size], out[k.size:]
