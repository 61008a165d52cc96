"""ctypes wrapper over the CPU oracle (oracle/tpm_oracle.cpp).

TEST INFRASTRUCTURE ONLY: the CPU restatement of the reference PME kick path
that the CUDA product is checked against, and the CPU baseline that bench.py
times.  Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import
this module; the product package never does.

Each wrapper names the reference function it restates (paths relative to the
dmarce1/tigerpm tree); the C++ file cites the exact lines.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")


class KickParams(C.Structure):
    _fields_ = [
        ("N", C.c_int), ("C", C.c_int), ("rs", C.c_double), ("GM", C.c_double),
        ("eta", C.c_double), ("hsoft", C.c_double), ("rcut", C.c_double),
        ("min_rung", C.c_int), ("scale", C.c_double), ("t0", C.c_double),
        ("first_call", C.c_int), ("precision", C.c_int),
    ]


def build() -> str:
    """Compile liboracle.so with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "tpm_oracle.cpp")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        build()
    L = C.CDLL(path)
    L.orc_fixed32_from_double.restype = C.c_uint32
    L.orc_fixed32_from_double.argtypes = [C.c_double]
    L.orc_fixed32_to_float.restype = C.c_float
    L.orc_fixed32_to_float.argtypes = [C.c_uint32]
    L.orc_fixed32_to_double.restype = C.c_double
    L.orc_fixed32_to_double.argtypes = [C.c_uint32]
    L.orc_distance.restype = C.c_float
    L.orc_distance.argtypes = [C.c_uint32, C.c_uint32]
    L.orc_erfcexp.restype = C.c_float
    L.orc_erfcexp.argtypes = [C.c_float, C.POINTER(C.c_float)]
    L.orc_fixed32_from_double_array.argtypes = [C.c_int64, f64p, u32p]
    L.orc_fixed32_convert_array.argtypes = [C.c_int64, u32p, u32p, f32p, f64p, f32p]
    L.orc_cloud4_array.argtypes = [C.c_int64, f64p, f64p]
    L.orc_mesh_loc.argtypes = [C.c_int, C.c_int64, u32p, i32p]
    L.orc_chainmesh_sort.restype = C.c_int
    L.orc_chainmesh_sort.argtypes = [C.c_int, C.c_int64, u32p, u32p, u32p, f32p, f32p, f32p,
                                     i8p, i32p, i32p, C.c_int]
    L.orc_deposit.restype = C.c_int
    L.orc_deposit.argtypes = [C.c_int, C.c_int, C.c_int64, u32p, u32p, u32p, f64p, C.c_int]
    L.orc_fft3d_r2c.argtypes = [C.c_int, f64p, f64p]
    L.orc_fft3d_c2r.argtypes = [C.c_int, f64p, f64p]
    L.orc_green_apply.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, f64p]
    L.orc_gravity_long.restype = C.c_int
    L.orc_gravity_long.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int64,
                                   u32p, u32p, u32p, f64p, C.c_int]
    L.orc_kick_pme.restype = C.c_int
    L.orc_kick_pme.argtypes = [C.POINTER(KickParams), C.c_int64, u32p, u32p, u32p, f32p, f32p,
                               f32p, i8p, i32p, i32p, C.c_void_p, C.c_void_p, f32p, f32p, f32p,
                               f32p, C.c_void_p, C.c_int64, i64p, C.c_int]
    L.orc_ewald_ref.argtypes = [C.c_int64, u32p, u32p, u32p, C.c_int64, u32p, u32p, u32p,
                                C.c_double, f64p, f64p, f64p, f64p, C.c_int]
    L.orc_drift.restype = C.c_int
    L.orc_drift.argtypes = [C.c_int64, u32p, u32p, u32p, f32p, f32p, f32p, C.c_double]
    L.orc_max_threads.restype = C.c_int
    _LIB = L
    return L


# ------------------------------------------------------------------ fixed32

def fixed32_from_double(x: float) -> int:
    """fixed<uint32_t>(double) (tigerpm/fixed.hpp:63-75)."""
    return int(lib().orc_fixed32_from_double(float(x)))


def fixed32_to_float(i: int) -> float:
    """fixed::to_float (tigerpm/fixed.hpp:115-118)."""
    return float(lib().orc_fixed32_to_float(int(i)))


def fixed32_to_double(i: int) -> float:
    return float(lib().orc_fixed32_to_double(int(i)))


def distance(a: int, b: int) -> float:
    """distance(fixed32, fixed32) (tigerpm/gravity_short.hpp:20-22)."""
    return float(lib().orc_distance(int(a), int(b)))


def fixed32_from_double_array(x) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float64)
    out = np.empty(x.size, np.uint32)
    lib().orc_fixed32_from_double_array(x.size, x, out)
    return out


def fixed32_convert_array(a, b):
    """(to_float(a), to_double(a), distance(a, b)) elementwise."""
    a = np.ascontiguousarray(a, np.uint32)
    b = np.ascontiguousarray(b, np.uint32)
    tf = np.empty(a.size, np.float32)
    td = np.empty(a.size, np.float64)
    ds = np.empty(a.size, np.float32)
    lib().orc_fixed32_convert_array(a.size, a, b, tf, td, ds)
    return tf, td, ds


def cloud4(x) -> np.ndarray:
    """cloud4 (src/gravity_long.cpp:127-138)."""
    x = np.ascontiguousarray(x, np.float64)
    out = np.empty(x.size, np.float64)
    lib().orc_cloud4_array(x.size, x, out)
    return out


def erfcexp(x: float):
    e = C.c_float()
    r = lib().orc_erfcexp(float(x), C.byref(e))
    return float(r), float(e.value)


def mesh_loc(C_: int, x: np.ndarray) -> np.ndarray:
    """particles_mesh_loc for one coordinate (tigerpm/particles.hpp:60-67)."""
    x = np.ascontiguousarray(x, np.uint32)
    out = np.empty(x.size, np.int32)
    lib().orc_mesh_loc(C_, x.size, x, out)
    return out


# ---------------------------------------------------------------- particles

@dataclass
class Particles:
    """Host SoA particle store (src/particles.cpp:6-12)."""
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray
    rung: np.ndarray

    @property
    def n(self) -> int:
        return int(self.x.size)

    def copy(self) -> "Particles":
        return Particles(*(np.array(a, copy=True) for a in
                           (self.x, self.y, self.z, self.vx, self.vy, self.vz, self.rung)))


def chainmesh_sort(C_: int, p: Particles, nthreads: int = 0):
    """chainmesh_create on one rank: in-place partition sort of p; returns
    (pbegin, pend) keyed (z*C+y)*C+x (src/chainmesh.cpp:139-213)."""
    nc = C_ ** 3
    pb = np.empty(nc, np.int32)
    pe = np.empty(nc, np.int32)
    rc = lib().orc_chainmesh_sort(C_, p.n, p.x, p.y, p.z, p.vx, p.vy, p.vz, p.rung, pb, pe,
                                  nthreads)
    if rc:
        raise ValueError("orc_chainmesh_sort failed")
    return pb, pe


def deposit(N: int, assign: int, x, y, z, nthreads: int = 0) -> np.ndarray:
    """compute_source (src/gravity_long.cpp:142-199) -> float64 N^3 grid."""
    rho = np.empty(N ** 3, np.float64)
    rc = lib().orc_deposit(N, assign, x.size, x, y, z, rho, nthreads)
    if rc:
        raise ValueError("orc_deposit failed")
    return rho.reshape(N, N, N)


def fft3d_r2c(rho: np.ndarray) -> np.ndarray:
    N = rho.shape[0]
    out = np.empty(N * N * (N // 2 + 1) * 2, np.float64)
    lib().orc_fft3d_r2c(N, np.ascontiguousarray(rho, np.float64).ravel(), out)
    return out.view(np.complex128).reshape(N, N, N // 2 + 1)


def fft3d_c2r(Y: np.ndarray) -> np.ndarray:
    N = Y.shape[0]
    buf = np.ascontiguousarray(Y, np.complex128).copy().view(np.float64).ravel()
    out = np.empty(N ** 3, np.float64)
    lib().orc_fft3d_c2r(N, buf, out)
    return out.reshape(N, N, N)


def green_apply(Y: np.ndarray, rs_cells: float, pme: int = 1, deconv_order: int = 4) -> np.ndarray:
    """apply_laplacian (src/gravity_long.cpp:201-245) on a copy of Y."""
    N = Y.shape[0]
    buf = np.ascontiguousarray(Y, np.complex128).copy()
    flat = buf.view(np.float64).ravel()
    lib().orc_green_apply(N, rs_cells, pme, deconv_order, flat)
    return flat.view(np.complex128).reshape(Y.shape)


def gravity_long(N: int, rs_cells: float, assign: int, x, y, z, pme: int = 1,
                 deconv_order: int | None = None, nthreads: int = 0) -> np.ndarray:
    """gravity_long_compute (src/gravity_long.cpp:36-48): periodic phi, float64."""
    if deconv_order is None:
        deconv_order = {0: 4, 1: 2, 2: 3}[assign]
    phi = np.empty(N ** 3, np.float64)
    rc = lib().orc_gravity_long(N, rs_cells, pme, assign, deconv_order, x.size, x, y, z, phi,
                                nthreads)
    if rc:
        raise ValueError("orc_gravity_long failed")
    return phi.reshape(N, N, N)


def kick_pme(params: KickParams, p: Particles, pbegin, pend, phi, sink_cells=None,
             nthreads: int = 0):
    """kick_pme_kernel restated (src/kick_pme.cu:128-357).  Updates p.vx/vy/vz/
    rung in place; returns (gx, gy, gz, pot, pair_counts, n_rung_errors)."""
    n = p.n
    gx = np.zeros(n, np.float32)
    gy = np.zeros(n, np.float32)
    gz = np.zeros(n, np.float32)
    pot = np.zeros(n, np.float32)
    counts = np.zeros(2, np.int64)
    phi = np.ascontiguousarray(phi)
    pf = phi.ctypes.data if phi.dtype == np.float32 else None
    pd = phi.ctypes.data if phi.dtype == np.float64 else None
    if sink_cells is None:
        sc, nsc = None, -1
    else:
        sink_cells = np.ascontiguousarray(sink_cells, np.int32)
        sc, nsc = sink_cells.ctypes.data, sink_cells.size
    bad = lib().orc_kick_pme(C.byref(params), n, p.x, p.y, p.z, p.vx, p.vy, p.vz, p.rung,
                             pbegin, pend, pf, pd, gx, gy, gz, pot, sc, nsc, counts, nthreads)
    return gx, gy, gz, pot, counts, bad


def ewald_ref(x, y, z, sx, sy, sz, hsoft: float, nthreads: int = 0):
    """gravity_ewald_kernel structure in FP64 (src/gravity_short.cu:93-201)."""
    s = sx.size
    phi = np.empty(s)
    gx = np.empty(s)
    gy = np.empty(s)
    gz = np.empty(s)
    lib().orc_ewald_ref(x.size, x, y, z, s, np.ascontiguousarray(sx, np.uint32),
                        np.ascontiguousarray(sy, np.uint32), np.ascontiguousarray(sz, np.uint32),
                        hsoft, phi, gx, gy, gz, nthreads)
    return phi, gx, gy, gz


def drift(p: Particles, dt: float) -> None:
    rc = lib().orc_drift(p.n, p.x, p.y, p.z, p.vx, p.vy, p.vz, float(dt))
    if rc:
        raise ValueError("orc_drift: |v*dt| too large")


def max_threads() -> int:
    return int(lib().orc_max_threads())


# ------------------------------------------------------- initial conditions

def philox4x32_10(ctr, key):
    """Philox-4x32-10 (Salmon et al. SC'11) of one 4-word counter, 2-word key."""
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    out = np.empty(4, np.uint32)
    L = lib()
    L.orc_philox4x32_10.argtypes = [u32p, u32p, u32p]
    L.orc_philox4x32_10(c, k, out)
    return out


def ic_power(table_k, table_p, hubble: float, sigma8: float, k):
    """power_spectrum_function (src/initialize.cpp:10-66,182-211) at k (1/Mpc)."""
    tk = np.ascontiguousarray(table_k, np.float64)
    tp = np.ascontiguousarray(table_p, np.float64)
    k = np.ascontiguousarray(k, np.float64)
    out = np.empty(k.size)
    L = lib()
    L.orc_ic_power.restype = C.c_int
    L.orc_ic_power.argtypes = [f64p, f64p, C.c_int, C.c_double, C.c_double, C.c_int64, f64p, f64p]
    if L.orc_ic_power(tk, tp, tk.size, hubble, sigma8, k.size, k, out):
        raise ValueError("orc_ic_power failed")
    return out


def growth_factor(omega_m: float, a: float) -> float:
    """growth_factor (src/initialize.cpp:76-83)."""
    L = lib()
    L.orc_growth_factor.restype = C.c_double
    L.orc_growth_factor.argtypes = [C.c_double, C.c_double]
    return float(L.orc_growth_factor(omega_m, a))


def ic_zeldovich(N: int, seed: int, table_k=None, table_p=None, index: float = -2.0, kcut: float = 0.5,
                 rms_disp: float = 0.0, hubble: float = 0.7, sigma8: float = 0.84, code_to_cm: float = 0.0,
                 omega_m: float = 0.3, z0: float = 2.0):
    """zeldovich_begin / fft3d_force_real / zeldovich_end (src/initialize.cpp:91-180)
    in FP64 with Philox deviates; returns (x, y, z) fixed32 and max |dx| N."""
    n = N ** 3
    x = np.empty(n, np.uint32)
    y = np.empty(n, np.uint32)
    z = np.empty(n, np.uint32)
    dmax = C.c_double()
    if table_k is None:
        tk = tp = np.zeros(1)
        npow = 0
    else:
        tk = np.ascontiguousarray(table_k, np.float64)
        tp = np.ascontiguousarray(table_p, np.float64)
        npow = tk.size
    L = lib()
    L.orc_ic_zeldovich.restype = C.c_int
    L.orc_ic_zeldovich.argtypes = [C.c_int, C.c_uint64, C.c_int, f64p, f64p, C.c_double, C.c_double, C.c_double,
                                   C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, u32p, u32p, u32p,
                                   C.POINTER(C.c_double)]
    if L.orc_ic_zeldovich(N, seed, npow, tk, tp, index, kcut, rms_disp, hubble, sigma8, code_to_cm, omega_m, z0,
                          x, y, z, C.byref(dmax)):
        raise ValueError("orc_ic_zeldovich failed")
    return x, y, z, float(dmax.value)
