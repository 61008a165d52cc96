"""Shared helpers for the parity tests: build a box on the device and the
same box in the oracle from one seeded particle set."""
from __future__ import annotations

import math

import numpy as np

from tigerpm_b200 import workloads as W


def particle_set(kind: str, n_side: int, seed: int, grid: int | None = None):
    if kind == "uniform":
        return W.uniform(n_side ** 3, seed)
    if kind == "zeldovich":
        return W.zeldovich(n_side, seed, grid=grid or n_side)
    if kind == "halos":
        return W.nfw_halos(n_side, seed, n_halo=max(4, n_side), halo_frac=0.7)
    raise ValueError(kind)


def with_random_motion(ps, seed: int, vscale: float = 1e-3, max_rung: int = 3):
    g = W.rng(seed + 99)
    n = ps.n
    ps.vx[:] = g.normal(0, vscale, n).astype(np.float32)
    ps.vy[:] = g.normal(0, vscale, n).astype(np.float32)
    ps.vz[:] = g.normal(0, vscale, n).astype(np.float32)
    ps.rung[:] = g.integers(0, max_rung + 1, n).astype(np.int8)
    return ps


def oracle_particles(O, ps):
    return O.Particles(*(np.array(a, copy=True) for a in ps.arrays()))


def kick_params(O, opts, min_rung=0, scale=1.0, t0=1.0, first_call=True, precision=0):
    rcut = opts.rcut_over_rs * opts.rs if opts.rcut_over_rs > 0 else 0.0
    return O.KickParams(N=opts.four_dim, C=opts.chain_dim, rs=opts.rs, GM=opts.GM, eta=opts.eta,
                        hsoft=opts.hsoft, rcut=rcut, min_rung=min_rung, scale=scale, t0=t0,
                        first_call=1 if first_call else 0, precision=precision)


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return math.sqrt(float(np.sum((a - b) ** 2)) / max(float(np.sum(b * b)), 1e-300))
