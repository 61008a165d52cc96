"""Seeded synthetic particle sets for the PME kick.

All generators draw from numpy's Philox-4x32-10 counter-based generator
(Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as easy as 1, 2, 3",
SC'11), so a (kind, size, seed) triple names one input exactly.  Positions are
returned as the reference's 32-bit fixed point: raw = floor(x * 2^32) for
x in [0, 1) (tigerpm/fixed.hpp:63-75), velocities float32, rungs int8.

The shapes follow the reference's own test inputs (uniform random positions,
zero velocities and rungs, src/particles.cpp:100-132) and the clustered
Zel'dovich / halo inputs the benchmark configurations name.  The reference
draws with GSL's taus generator; that stream is not reproduced, so "same seed"
means the same Philox stream here on both sides of every comparison.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

TWO32 = 4294967296.0


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(int(seed)))


@dataclass
class ParticleSet:
    """Host SoA particle arrays (the reference's particles_X/U/R)."""
    x: np.ndarray  # uint32 fixed point
    y: np.ndarray
    z: np.ndarray
    vx: np.ndarray  # float32
    vy: np.ndarray
    vz: np.ndarray
    rung: np.ndarray  # int8

    @property
    def n(self) -> int:
        return int(self.x.size)

    def copy(self) -> "ParticleSet":
        return ParticleSet(*(np.array(a, copy=True) for a in self.arrays()))

    def arrays(self):
        return (self.x, self.y, self.z, self.vx, self.vy, self.vz, self.rung)


def _from_positions(pos: np.ndarray) -> ParticleSet:
    """pos: float64 (3, n) in box units, wrapped into [0, 1)."""
    pos = np.mod(pos, 1.0)
    raw = np.floor(pos * TWO32)
    raw = np.minimum(raw, TWO32 - 1).astype(np.uint32)
    n = pos.shape[1]
    z32 = np.zeros(n, np.float32)
    return ParticleSet(np.ascontiguousarray(raw[0]), np.ascontiguousarray(raw[1]),
                       np.ascontiguousarray(raw[2]), z32.copy(), z32.copy(), z32.copy(),
                       np.zeros(n, np.int8))


def uniform(n: int, seed: int) -> ParticleSet:
    """n particles uniform in the periodic unit box, raw uint32 drawn directly."""
    g = rng(seed)
    raw = g.integers(0, 1 << 32, size=(3, n), dtype=np.uint64).astype(np.uint32)
    z32 = np.zeros(n, np.float32)
    return ParticleSet(np.ascontiguousarray(raw[0]), np.ascontiguousarray(raw[1]),
                       np.ascontiguousarray(raw[2]), z32.copy(), z32.copy(), z32.copy(),
                       np.zeros(n, np.int8))


def zeldovich(n_side: int, seed: int, rms_cells: float = 0.3, spectral_index: float = -2.0,
              kcut_over_nyq: float = 0.5, grid: int | None = None) -> ParticleSet:
    """n_side^3 particles on a lattice, displaced by the Zel'dovich field of a
    Gaussian random field with P(k) ~ k^n exp(-k / (kcut_over_nyq * k_Nyq))
    (the reading of "exponentially cut" used here), normalised so the rms
    3-D displacement is rms_cells mesh cells of a grid^3 mesh."""
    grid = n_side if grid is None else grid
    g = rng(seed)
    n = n_side
    white = g.standard_normal((n, n, n))
    dk = np.fft.rfftn(white)
    kx = np.fft.fftfreq(n) * n
    kz = np.fft.rfftfreq(n) * n
    KX, KY, KZ = np.meshgrid(kx, kx, kz, indexing="ij")
    k2 = KX * KX + KY * KY + KZ * KZ
    k = np.sqrt(k2)
    k_nyq = n / 2.0
    with np.errstate(divide="ignore", invalid="ignore"):
        amp = np.where(k > 0, k ** (spectral_index / 2.0) * np.exp(-k / (2.0 * kcut_over_nyq * k_nyq)), 0.0)
        inv_k2 = np.where(k2 > 0, 1.0 / k2, 0.0)
    dk *= amp
    disp = np.empty((3, n, n, n))
    for d, K in enumerate((KX, KY, KZ)):
        disp[d] = np.fft.irfftn(1j * K * inv_k2 * dk, s=(n, n, n), axes=(0, 1, 2))
    rms = math.sqrt(float(np.mean(np.sum(disp * disp, axis=0))))
    disp *= (rms_cells / grid) / rms
    q = (np.arange(n) + 0.5) / n
    QX, QY, QZ = np.meshgrid(q, q, q, indexing="ij")
    pos = np.stack([QX + disp[0], QY + disp[1], QZ + disp[2]]).reshape(3, -1)
    return _from_positions(pos)


def _nfw_mu(s):
    return np.log1p(s) - s / (1.0 + s)


def nfw_halos(n_side: int, seed: int, n_halo: int = 2000, halo_frac: float = 0.7,
              c_range=(5.0, 15.0), mass_decades: float = 3.0) -> ParticleSet:
    """halo_frac of n_side^3 particles in n_halo NFW halos (log-uniform masses
    over mass_decades, concentration uniform in c_range, centres uniform,
    r200 from 200x the mean density, radii by inverse NFW mass CDF), the rest
    uniform background."""
    g = rng(seed)
    N = n_side ** 3
    n_h = int(round(halo_frac * N))
    logm = g.uniform(0.0, mass_decades * math.log(10.0), n_halo)
    w = np.exp(logm)
    counts = np.floor(w / w.sum() * n_h).astype(np.int64)
    counts[: n_h - counts.sum()] += 1
    centres = g.uniform(0.0, 1.0, (n_halo, 3))
    conc = g.uniform(c_range[0], c_range[1], n_halo)
    r200 = np.cbrt(3.0 * counts / (800.0 * math.pi * N))
    hid = np.repeat(np.arange(n_halo), counts)
    c = conc[hid]
    u = g.uniform(0.0, 1.0, hid.size) * _nfw_mu(c)
    s = np.full(hid.size, 1.0)
    lo = np.zeros(hid.size)
    hi = c.copy()
    for _ in range(60):  # bisection on mu(s) = u, s in [0, c]
        s = 0.5 * (lo + hi)
        m = _nfw_mu(s) < u
        lo = np.where(m, s, lo)
        hi = np.where(m, hi, s)
    r = s / c * r200[hid]
    v = g.standard_normal((3, hid.size))
    v /= np.linalg.norm(v, axis=0)
    halo_pos = centres[hid].T + v * r
    bg = g.uniform(0.0, 1.0, (3, N - n_h))
    return _from_positions(np.concatenate([halo_pos, bg], axis=1))


def sample_indices(n: int, count: int, seed: int) -> np.ndarray:
    """Distinct particle indices for the Ewald comparison (the reference draws
    with rand() and drops duplicates, src/particles.cpp:333-381)."""
    count = min(count, n)
    return np.sort(rng(seed + 0x5EED).choice(n, size=count, replace=False)).astype(np.int64)


def log_uniform_sides(count: int, lo: int, hi: int, seed: int) -> np.ndarray:
    """Box sides n = round(exp(U[ln lo, ln hi])) for the batched / served pools."""
    g = rng(seed)
    return np.rint(np.exp(g.uniform(math.log(lo), math.log(hi), count))).astype(np.int64)


def fft_friendly(n_min: int) -> int:
    """Smallest mesh side >= n_min that the library's own FFT takes: a
    multiple of 16 whose cofactor has no prime factor above 5."""
    m = max(16, (int(n_min) + 15) // 16 * 16)
    while True:
        k = m // 16
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1:
            return m
        m += 16


def accurate_box_params(n_side: int) -> dict:
    """Mesh and split parameters of a box of n_side^3 particles in the form
    that meets rms force error <= 1e-4 against FP64 Ewald: the reference's
    cloud4 deposit on a mesh of at least 3 points per particle spacing
    (rounded up to a size the library's FFT takes), split scale r_s = 2/3
    particle spacing and cutoff 6 r_s = 4 particle spacings (64 particles
    per chain cell on average)."""
    grid = fft_friendly(3 * n_side)
    rs_cells = 2.0 * grid / (3.0 * n_side)
    return dict(n_side=n_side, grid=grid, rs_cells=rs_cells, rcut_over_rs=6.0, assign="cloud4")


def ensemble(count: int, lo: int, hi: int, seed: int, rms_cells: float = 0.3):
    """The batched / served pools: `count` Zel'dovich boxes (P(k) ~ k^-2 cut
    at k_Nyq/2, rms displacement rms_cells particle spacings) with sides
    log-uniform in [lo, hi] and per-box seeds.  Returns (sides, [ParticleSet])."""
    sides = log_uniform_sides(count, lo, hi, seed)
    sets = [zeldovich(int(n), seed * 1000 + i + 1, rms_cells=rms_cells, grid=int(n)) for i, n in enumerate(sides)]
    return sides, sets
