"""Zel'dovich initial conditions (src/initialize.cpp:10-221).

CPU: the oracle's power_spectrum_function / growth_factor restatement and
the library's host-side copies of them against golden vectors from the
reference's own reader, interpolation, sigma8 normalisation and growth
factor (tests/golden/ic_power.npz); Philox-4x32-10 against the published
known-answer vectors of Salmon et al.
GPU: the device generator (tpm_ic_zeldovich) against the oracle's FP64
restatement with the same deviates, for both spectrum forms."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from golden_io import load
from helpers import rel_rms


def test_philox_known_answers():
    kat = [([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
           ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
           ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
            [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1])]
    for ctr, key, want in kat:
        assert list(O.philox4x32_10(ctr, key)) == want


def _in_table(d):
    # inside the table's k range; outside it the reference extrapolates a
    # float cubic in ln k far from its nodes, where float rounding dominates
    h = float(d["hubble"])
    return (d["k"] >= d["table_k"].min() * h) & (d["k"] <= d["table_k"].max() * h)


def test_oracle_power_and_growth_vs_reference():
    d = load("ic_power")
    p = O.ic_power(d["table_k"], d["table_p"], float(d["hubble"]), float(d["sigma8"]), d["k"])
    m = _in_table(d)
    assert np.max(np.abs(p[m] / d["P"][m] - 1)) < 2e-5
    assert np.max(np.abs(p / d["P"] - 1)) < 2e-2
    g = np.array([O.growth_factor(a, b) for a, b in d["omega_a"]])
    assert np.max(np.abs(g / d["growth"] - 1)) < 1e-7


def test_library_power_and_growth_vs_reference(lib):
    d = load("ic_power")
    tk = np.ascontiguousarray(d["table_k"])
    tp = np.ascontiguousarray(d["table_p"])
    k = np.ascontiguousarray(d["k"])
    out = np.empty(k.size)
    f64 = lambda a: a.ctypes.data_as(C.c_void_p)
    rc = lib.tpm_ic_power(f64(tk), f64(tp), tk.size, float(d["hubble"]), float(d["sigma8"]), k.size, f64(k), f64(out))
    assert rc == 0
    m = _in_table(d)
    assert np.max(np.abs(out[m] / d["P"][m] - 1)) < 2e-5
    for (om, a), want in zip(d["omega_a"], d["growth"]):
        v = C.c_double()
        assert lib.tpm_growth_factor(float(om), float(a), C.byref(v)) == 0
        assert abs(v.value / want - 1) < 1e-7


def test_oracle_ic_statistics():
    """The FP64 generator's displacements: rms as requested, zero mean."""
    N = 20
    x, y, z, dmax = O.ic_zeldovich(N, 11, rms_disp=0.3)
    q = (np.arange(N) + 0.5) / N
    QX, QY, QZ = np.meshgrid(q, q, q, indexing="ij")
    d = []
    for a, Q in zip((x, y, z), (QX, QY, QZ)):
        v = a.astype(np.float64) / 2 ** 32 - Q.ravel()
        d.append((v + 0.5) % 1.0 - 0.5)
    d = np.stack(d) * N
    assert abs(np.sqrt(np.mean(np.sum(d * d, axis=0))) - 0.3) < 1e-6
    assert np.max(np.abs(np.mean(d, axis=1))) < 1e-8  # fixed32 truncation: half a unit of 2^-32
    assert abs(dmax - np.max(np.abs(d))) < 1e-6


def _device_ic(N, seed, **kw):
    from tigerpm_b200.api import TigerPM, make_options, ic_zeldovich
    opts = make_options(N, N, rs_cells=1.0)
    with TigerPM(opts, N ** 3) as t:
        dmax = ic_zeldovich(t, N, seed, **kw)
        x, y, z, vx, vy, vz, r = t.get_particles()
    assert not np.any(vx) and not np.any(r)
    return x, y, z, dmax, opts


def _max_units(a, b):
    return int(np.max(np.abs((a.astype(np.int64) - b.astype(np.int64) + 2 ** 31) % 2 ** 32 - 2 ** 31)))


@pytest.mark.gpu
@pytest.mark.parametrize("N,seed", [(16, 1), (33, 7), (48, 3)])
def test_device_ic_power_law_matches_oracle(N, seed):
    x, y, z, dmax, _ = _device_ic(N, seed, rms_disp=0.3)
    ox, oy, oz, odmax = O.ic_zeldovich(N, seed, rms_disp=0.3)
    # FP32 inverse FFT against FP64: a few units of 2^-32 of a displacement
    # of ~0.3 / N box lengths
    for a, b in ((x, ox), (y, oy), (z, oz)):
        assert _max_units(a, b) < 4096
    assert abs(dmax - odmax) < 1e-4 * odmax


@pytest.mark.gpu
def test_device_ic_reference_spectrum_matches_oracle():
    d = load("ic_power")
    N = 32
    x, y, z, dmax, opts = _device_ic(N, 5, table_k=d["table_k"], table_p=d["table_p"])
    ox, oy, oz, odmax = O.ic_zeldovich(N, 5, table_k=d["table_k"], table_p=d["table_p"], hubble=opts.hubble,
                                       sigma8=opts.sigma8, code_to_cm=opts.code_to_cm, omega_m=opts.omega_m,
                                       z0=opts.z0)
    for a, b in ((x, ox), (y, oy), (z, oz)):
        assert _max_units(a, b) < 4096
    assert abs(dmax - odmax) < 1e-4 * max(odmax, 1e-6)
