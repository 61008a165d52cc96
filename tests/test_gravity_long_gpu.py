"""Device long-range solve vs the oracle's restatement of
gravity_long_compute (src/gravity_long.cpp:36-256): deposit, FFT,
Green's function, inverse FFT; plus the phi read-out and force_at."""
import math

import numpy as np
import pytest

import oracle as O
from helpers import particle_set, rel_rms
from tigerpm_b200.api import GRAVITY_LONG_PM, GRAVITY_LONG_PME, Range, TigerPM, make_options

pytestmark = pytest.mark.gpu

ASSIGN_ID = {"cloud4": 0, "cic": 1, "tsc": 2}


def device_phi(ps, grid, assign, rs_cells, typ, chain=3, exact=0, fft="auto"):
    opts = make_options(round(ps.n ** (1 / 3)), grid, chain=chain, rs_cells=rs_cells, assign=assign,
                        deterministic_deposit=exact, fft=fft)
    with TigerPM(opts, ps.n) as t:
        t.set_particles(ps)
        t.chainmesh_create()
        t.gravity_long_compute(typ)
        phi = t.gravity_long_get_phi(Range((0, 0, 0), (grid, grid, grid)))
        x, y, z, *_ = t.get_particles()
    return phi, (x, y, z)


@pytest.mark.parametrize("assign", ["cloud4", "cic", "tsc"])
@pytest.mark.parametrize("grid,n_side", [(32, 24), (30, 20), (45, 16), (200, 40)])
@pytest.mark.parametrize("exact", [0, 1, 2])
def test_phi_matches_oracle(assign, grid, n_side, exact):
    ps = particle_set("uniform", n_side, 3)
    for typ in (GRAVITY_LONG_PME, GRAVITY_LONG_PM):
        phi, (x, y, z) = device_phi(ps, grid, assign, 1.25, typ, exact=exact)
        ref = O.gravity_long(grid, 1.25, ASSIGN_ID[assign], x, y, z, pme=typ)
        assert rel_rms(phi, ref) < 2e-6, (assign, grid, typ, rel_rms(phi, ref))


def test_deposit_mass_and_determinism():
    """Deposit is exact fixed-point: two runs give identical bits, and the
    k = 0 mode of the PM solve is removed (phi has zero mean)."""
    ps = particle_set("halos", 24, 5)
    a, _ = device_phi(ps, 32, "cloud4", 1.0, GRAVITY_LONG_PME, exact=True)
    b, _ = device_phi(ps, 32, "cloud4", 1.0, GRAVITY_LONG_PME, exact=True)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert abs(float(np.mean(a.astype(np.float64)))) < 1e-4 * float(np.abs(a).max())


def test_fixed32_deposit_is_bit_reproducible():
    """deterministic_deposit = 2 accumulates 26-bit fixed point with integer
    adds: repeated runs give identical bits, and phi agrees with the exact
    int64 deposit."""
    ps = particle_set("uniform", 24, 5)
    a, _ = device_phi(ps, 32, "cloud4", 1.0, GRAVITY_LONG_PME, exact=2)
    b, _ = device_phi(ps, 32, "cloud4", 1.0, GRAVITY_LONG_PME, exact=2)
    c, _ = device_phi(ps, 32, "cloud4", 1.0, GRAVITY_LONG_PME, exact=1)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert rel_rms(a, c) < 1e-6, rel_rms(a, c)


@pytest.mark.parametrize("assign", ["cloud4", "cic", "tsc"])
def test_dense_clump_deposit_matches_oracle(assign):
    """2,000 particles inside one quarter mesh cell put hundreds of weight
    units on a few points: with deterministic_deposit = 2 the fixed-point
    tiles there overflow their range and are deposited again in FP32; phi
    matches the oracle in every mode."""
    ps = particle_set("uniform", 16, 7)
    g = np.random.default_rng(3)
    k = 2000
    for arr in (ps.x, ps.y, ps.z):
        arr[:k] = np.uint32(1 << 31) + g.integers(0, 1 << 25, k).astype(np.uint32)
    for exact in (0, 1, 2):
        phi, (x, y, z) = device_phi(ps, 32, assign, 1.25, GRAVITY_LONG_PME, exact=exact)
        ref = O.gravity_long(32, 1.25, ASSIGN_ID[assign], x, y, z, pme=GRAVITY_LONG_PME)
        assert rel_rms(phi, ref) < 2e-6, (assign, exact, rel_rms(phi, ref))


def test_get_phi_periodic_box():
    ps = particle_set("uniform", 16, 4)
    grid = 16
    opts = make_options(16, grid, chain=3, rs_cells=1.0)
    with TigerPM(opts, ps.n) as t:
        t.set_particles(ps)
        t.chainmesh_create()
        t.gravity_long_compute(GRAVITY_LONG_PME)
        full = t.gravity_long_get_phi(Range((0, 0, 0), (grid, grid, grid)))
        box = t.gravity_long_get_phi_box()
        assert box.begin == (-3, -3, -3) and box.end == (grid + 3,) * 3
        padded = t.gravity_long_get_phi(box)
        sub = t.gravity_long_get_phi(Range((5, -2, 14), (9, 3, 20)))
    idx = np.arange(-3, grid + 3) % grid
    assert np.array_equal(padded, full[np.ix_(idx, idx, idx)])
    ii = np.arange(5, 9) % grid
    jj = np.arange(-2, 3) % grid
    kk = np.arange(14, 20) % grid
    assert np.array_equal(sub, full[np.ix_(ii, jj, kk)])


def force_at_numpy(phi, pos):
    """gravity_long_force_at restated in numpy (src/gravity_long.cpp:52-125)."""
    N = phi.shape[0]
    out_p = np.empty(len(pos))
    out_g = np.empty((len(pos), 3))
    for n, p in enumerate(pos):
        X = np.array(p) * N
        I = X.astype(int)
        X = X - I
        I = I - 1
        w = np.stack([-0.5 * X + X ** 2 - 0.5 * X ** 3, 1 - 2.5 * X ** 2 + 1.5 * X ** 3,
                      0.5 * X + 2 * X ** 2 - 1.5 * X ** 3, -0.5 * X ** 2 + 0.5 * X ** 3], 1)
        dw = np.stack([-0.5 + 2 * X - 1.5 * X ** 2, -5 * X + 4.5 * X ** 2, 0.5 + 4 * X - 4.5 * X ** 2,
                       -X + 1.5 * X ** 2], 1)
        sub = phi[np.ix_((I[0] + np.arange(4)) % N, (I[1] + np.arange(4)) % N, (I[2] + np.arange(4)) % N)]
        out_p[n] = np.einsum("a,b,c,abc", w[0], w[1], w[2], sub)
        out_g[n, 0] = -np.einsum("a,b,c,abc", dw[0], w[1], w[2], sub) * N
        out_g[n, 1] = -np.einsum("a,b,c,abc", w[0], dw[1], w[2], sub) * N
        out_g[n, 2] = -np.einsum("a,b,c,abc", w[0], w[1], dw[2], sub) * N
    return out_p, out_g


def test_force_at():
    ps = particle_set("uniform", 16, 8)
    grid = 16
    opts = make_options(16, grid, chain=3, rs_cells=1.0)
    pos = np.random.default_rng(1).uniform(0, 1, (50, 3))
    with TigerPM(opts, ps.n) as t:
        t.set_particles(ps)
        t.chainmesh_create()
        t.gravity_long_compute(GRAVITY_LONG_PM)
        full = t.gravity_long_get_phi(Range((0, 0, 0), (grid, grid, grid))).astype(np.float64)
        p, g = t.gravity_long_force_at(pos)
    rp, rg = force_at_numpy(full, pos)
    assert rel_rms(p, rp) < 1e-6 and rel_rms(g, rg) < 1e-6


# The library's own transforms (fft3d.cu) run for grids that are multiples of
# 16 made of the radices 16, 8, 4, 3, 5 and 2: the generic block engine for
# every such grid (fft="block"), the warp-per-line engine by default where the
# grid has a compiled line plan (96, 128, 160 here; 48 and 80 have none and
# take the block engine).  Each is compared against both the oracle and cuFFT
# on the same deposit.
@pytest.mark.parametrize("fft", ["auto", "block"])
@pytest.mark.parametrize("grid", [48, 80, 96, 128, 160])
def test_library_fft_matches_oracle_and_cufft(grid, fft):
    ps = particle_set("uniform", 20, 4)
    for typ in (GRAVITY_LONG_PME, GRAVITY_LONG_PM):
        phi, (x, y, z) = device_phi(ps, grid, "cloud4", 2.0, typ, exact=True, fft=fft)
        phi_cu, _ = device_phi(ps, grid, "cloud4", 2.0, typ, exact=True, fft="cufft")
        ref = O.gravity_long(grid, 2.0, 0, x, y, z, pme=typ)
        assert rel_rms(phi, ref) < 2e-6, (grid, typ, rel_rms(phi, ref))
        assert rel_rms(phi, phi_cu) < 2e-6, (grid, typ, rel_rms(phi, phi_cu))


@pytest.mark.parametrize("grid", [64, 96, 128, 144, 160, 192, 240, 256, 288, 320, 384, 512, 576, 640])
def test_line_fft_engine_matches_block_engine_and_cufft(grid):
    """Every mesh with a compiled line plan (radix plans such as 12.8.8 at
    768, 12.8.4 at 384, 12.12 at 144, 10.6.2.2 at 240) against the generic
    block engine and cuFFT."""
    ps = particle_set("uniform", 24, 6)
    for typ in (GRAVITY_LONG_PME, GRAVITY_LONG_PM):
        phi, _ = device_phi(ps, grid, "cloud4", 2.0, typ, exact=True)
        phi_bl, _ = device_phi(ps, grid, "cloud4", 2.0, typ, exact=True, fft="block")
        phi_cu, _ = device_phi(ps, grid, "cloud4", 2.0, typ, exact=True, fft="cufft")
        assert rel_rms(phi, phi_bl) < 2e-6, (grid, typ, rel_rms(phi, phi_bl))
        assert rel_rms(phi, phi_cu) < 2e-6, (grid, typ, rel_rms(phi, phi_cu))


def test_library_fft_768_matches_cufft():
    """The benchmark mesh (768 = 4^4 x 3) against cuFFT on one deposit."""
    ps = particle_set("uniform", 64, 5)
    phi, _ = device_phi(ps, 768, "cloud4", 2.0, GRAVITY_LONG_PME, chain=64, exact=True)
    phi_cu, _ = device_phi(ps, 768, "cloud4", 2.0, GRAVITY_LONG_PME, chain=64, exact=True, fft="cufft")
    assert rel_rms(phi, phi_cu) < 2e-6, rel_rms(phi, phi_cu)
