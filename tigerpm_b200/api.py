"""Host-side mirror of the reference's PME-kick interface over the C ABI.

The reference exposes free C++ functions over global particle state
(tigerpm/kick_pme.hpp, chainmesh.hpp, gravity_long.hpp, gravity_short.hpp,
options.hpp).  `TigerPM` keeps one periodic box on the device and offers the
same operations under the same names, with the same argument meaning:

    chainmesh_create / chainmesh_get / chainmesh_interior_box
    gravity_long_compute / gravity_long_get_phi / gravity_long_get_phi_box /
        gravity_long_force_at
    kick_pme / kick_pme_begin / kick_pme_end
    gravity_short_ewald_call_kernel / gravity_short_ewald_compare
    drift (no reference counterpart)

Every call goes to libtigerpm_b200.so; failures raise TPMError carrying the
library's status and message (the reference prints and continues or aborts).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import GRAVITY_LONG_PM, GRAVITY_LONG_PME, Options, TPMError, check  # noqa: F401


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dataclass
class Range:
    """range<int> (tigerpm/range.hpp): half-open integer box, index() with z fastest."""
    begin: tuple
    end: tuple

    def volume(self) -> int:
        v = 1
        for b, e in zip(self.begin, self.end):
            if e < b:
                return 0
            v *= e - b
        return v

    def pad(self, dx: int = 1) -> "Range":
        return Range(tuple(b - dx for b in self.begin), tuple(e + dx for e in self.end))

    def shape(self):
        return tuple(e - b for b, e in zip(self.begin, self.end))

    def as_array(self):
        return (C.c_int * 6)(*self.begin, *self.end)


def options_for(parts_dim: int, parts_o_four: int = 3, four_o_chain: int = 5) -> Options:
    """process_options's derived values for the given sizes (src/options.cpp:81-96)."""
    lib = _lib.load()
    o = Options()
    check(lib.tpm_options_init(C.byref(o), parts_dim, parts_o_four, four_o_chain), "options_init")
    return o


def process_options(argv) -> Options:
    """Parse the reference's flags (--parts_dim, --parts_o_four, --four_o_chain,
    --box_size, --test, --config_file) plus the extensions listed in tpm.h."""
    lib = _lib.load()
    o = Options()
    arr = (C.c_char_p * len(argv))(*[a.encode() for a in argv])
    check(lib.tpm_options_parse(C.byref(o), len(argv), arr), "options_parse")
    return o


def make_options(n_side: int, grid: int, chain: int | None = None, rs_cells: float = 1.0,
                 rcut_over_rs: float = 0.0, assign: str = "cloud4", sort: str = "parity",
                 kahan: bool = True, GM: float = 1.0, deterministic_deposit: bool | int = False,
                 fft: str = "auto") -> Options:
    """Options for a box of n_side^3 particles on a grid^3 mesh.  chain=None
    picks the largest chain mesh whose cells are at least the cutoff wide
    (or rcut = 4.5 rs wide when there is no cutoff).  deterministic_deposit:
    False / 0 FP32 atomics, True / 1 exact int64, 2 26-bit fixed point."""
    o = options_for(n_side, 1, 1)
    o.four_dim = grid
    o.parts_o_four = 1
    o.rs = rs_cells / grid
    width = (rcut_over_rs if rcut_over_rs > 0 else 4.5) * rs_cells
    o.chain_dim = chain if chain is not None else max(3, int(grid / width))
    o.four_o_chain = max(1, grid // o.chain_dim)
    o.parts_o_chain = o.four_o_chain
    o.rcut_over_rs = rcut_over_rs
    o.assign = _lib.ASSIGN[assign]
    o.sort_mode = _lib.SORT[sort]
    o.kahan = 1 if kahan else 0
    o.deterministic_deposit = int(deterministic_deposit)
    o.fft = _lib.FFT[fft]
    o.GM = GM
    return o


def force_errors(g_test: np.ndarray, g_ref: np.ndarray, p_test=None, p_ref=None) -> dict:
    """gravity_short_ewald_compare's metrics (src/gravity_short.cpp:53-79):
    magnitude RMS sqrt(sum(|g1|-|g2|)^2 / sum|g2|^2), the reference's
    "max" sum||g1|-|g2|| / sqrt(sum|g2|^2), the same for phi, plus the vector
    RMS sqrt(sum|g1-g2|^2 / sum|g2|^2)."""
    g1 = np.asarray(g_test, np.float64)
    g2 = np.asarray(g_ref, np.float64)
    m1 = np.linalg.norm(g1, axis=1)
    m2 = np.linalg.norm(g2, axis=1)
    norm = float(np.sum(m2 * m2))
    out = {
        "force_rms_vector": math.sqrt(float(np.sum((g1 - g2) ** 2)) / norm),
        "force_rms": math.sqrt(float(np.sum((m1 - m2) ** 2)) / norm),
        "force_max": float(np.sum(np.abs(m1 - m2))) / math.sqrt(norm),
    }
    if p_test is not None and p_ref is not None:
        f1 = np.asarray(p_test, np.float64)
        f2 = np.asarray(p_ref, np.float64)
        pn = float(np.sum(f2 * f2))
        out["phi_rms"] = math.sqrt(float(np.sum((f1 - f2) ** 2)) / pn)
        out["phi_max"] = float(np.sum(np.abs(f1 - f2))) / math.sqrt(pn)
    return out


class TigerPM:
    """One periodic box resident on the current CUDA device."""

    def __init__(self, opts: Options, capacity: int):
        self.lib = _lib.load()
        self.opts = opts
        h = C.c_void_p()
        check(self.lib.tpm_ctx_create(C.byref(opts), int(capacity), C.byref(h)), "ctx_create")
        self.h = h
        self.capacity = int(capacity)
        self.n = 0
        self.owned = True

    @classmethod
    def borrow(cls, handle, opts: Options, n: int) -> "TigerPM":
        """A view of a context owned elsewhere (a batch's box); close() does
        not destroy it."""
        t = cls.__new__(cls)
        t.lib = _lib.load()
        t.opts = opts
        t.h = handle
        t.capacity = int(n)
        t.n = int(n)
        t.owned = False
        return t

    def close(self):
        if self.h and self.owned:
            self.lib.tpm_ctx_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------ particles
    def set_particles(self, ps) -> None:
        """particles_X/U/R <- ps (host arrays)."""
        x, y, z, vx, vy, vz, r = (np.ascontiguousarray(a) for a in
                                  (ps.x, ps.y, ps.z, ps.vx, ps.vy, ps.vz, ps.rung))
        assert x.dtype == np.uint32 and vx.dtype == np.float32 and r.dtype == np.int8
        check(self.lib.tpm_set_particles(self.h, x.size, _ptr(x), _ptr(y), _ptr(z), _ptr(vx), _ptr(vy),
                                         _ptr(vz), _ptr(r)), "set_particles")
        self.n = int(x.size)

    def set_particles_device(self, n: int, ptrs) -> None:
        """From device pointers (x, y, z, vx, vy, vz, rung) as ints."""
        check(self.lib.tpm_set_particles_device(self.h, int(n), *[C.c_void_p(p) for p in ptrs]),
              "set_particles_device")
        self.n = int(n)

    def get_particles(self):
        n = self.n
        x = np.empty(n, np.uint32)
        y = np.empty(n, np.uint32)
        z = np.empty(n, np.uint32)
        vx = np.empty(n, np.float32)
        vy = np.empty(n, np.float32)
        vz = np.empty(n, np.float32)
        r = np.empty(n, np.int8)
        check(self.lib.tpm_get_particles(self.h, _ptr(x), _ptr(y), _ptr(z), _ptr(vx), _ptr(vy), _ptr(vz),
                                         _ptr(r)), "get_particles")
        return x, y, z, vx, vy, vz, r

    def get_forces(self):
        """particles_G / particles_P of the last kick (FORCE_TEST)."""
        n = self.n
        g = [np.empty(n, np.float32) for _ in range(4)]
        check(self.lib.tpm_get_forces(self.h, *[_ptr(a) for a in g]), "get_forces")
        return g[0], g[1], g[2], g[3]

    def device_arrays(self) -> _lib.DeviceArrays:
        d = _lib.DeviceArrays()
        check(self.lib.tpm_get_device_arrays(self.h, C.byref(d)), "get_device_arrays")
        return d

    # ----------------------------------------------------------- chain mesh
    def chainmesh_create(self) -> None:
        check(self.lib.tpm_chainmesh_create(self.h), "chainmesh_create")

    def chainmesh_get(self, ijk):
        b = C.c_int32()
        e = C.c_int32()
        arr = (C.c_int * 3)(*ijk)
        check(self.lib.tpm_chainmesh_get(self.h, arr, C.byref(b), C.byref(e)), "chainmesh_get")
        return int(b.value), int(e.value)

    def chainmesh_offsets(self) -> np.ndarray:
        c = self.opts.chain_dim
        out = np.empty(c ** 3 + 1, np.int32)
        check(self.lib.tpm_chainmesh_offsets(self.h, _ptr(out)), "chainmesh_offsets")
        return out

    def chainmesh_interior_box(self) -> Range:
        b = (C.c_int * 6)()
        check(self.lib.tpm_chainmesh_interior_box(self.h, b), "chainmesh_interior_box")
        return Range(tuple(b[0:3]), tuple(b[3:6]))

    # ----------------------------------------------------------- long range
    def gravity_long_compute(self, type: int = GRAVITY_LONG_PM) -> None:
        check(self.lib.tpm_gravity_long_compute(self.h, int(type)), "gravity_long_compute")

    def gravity_long_get_phi(self, box: Range) -> np.ndarray:
        out = np.empty(box.volume(), np.float32)
        check(self.lib.tpm_gravity_long_get_phi(self.h, box.as_array(), _ptr(out)), "gravity_long_get_phi")
        return out.reshape(box.shape())

    def gravity_long_set_phi(self, phi: np.ndarray) -> None:
        """Load a periodic four_dim^3 potential (x-major, z fastest) computed
        elsewhere; kick_pme then uses it as gravity_long_get_phi's result."""
        a = np.ascontiguousarray(phi, np.float32)
        if a.size != self.opts.four_dim ** 3:
            raise ValueError("phi must hold four_dim^3 values")
        check(self.lib.tpm_gravity_long_set_phi(self.h, _ptr(a)), "gravity_long_set_phi")

    def gravity_long_get_phi_box(self) -> Range:
        b = (C.c_int * 6)()
        check(self.lib.tpm_gravity_long_get_phi_box(self.h, b), "gravity_long_get_phi_box")
        return Range(tuple(b[0:3]), tuple(b[3:6]))

    def gravity_long_force_at(self, pos: np.ndarray):
        """pos: (n, 3) float64 box units -> (phi[n], g[n, 3])."""
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
        n = pos.shape[0]
        phi = np.empty(n, np.float32)
        g = np.empty((n, 3), np.float32)
        check(self.lib.tpm_gravity_long_force_at(self.h, n, _ptr(pos), _ptr(phi), _ptr(g)),
              "gravity_long_force_at")
        return phi, g

    # ----------------------------------------------------------------- kick
    def kick_pme(self, box: Range | None, min_rung: int, scale: float, t0: float, first_call: bool) -> None:
        arr = box.as_array() if box is not None else None
        check(self.lib.tpm_kick_pme(self.h, arr, int(min_rung), float(scale), float(t0),
                                    1 if first_call else 0), "kick_pme")

    def kick_pme_begin(self, min_rung: int, scale: float, t0: float, first_call: bool) -> None:
        """kick_pme over chainmesh_interior_box() (src/kick_pme.cpp:9-18)."""
        self.kick_pme(self.chainmesh_interior_box(), min_rung, scale, t0, first_call)

    def kick_pme_end(self) -> None:
        """Drops ghost particles in the reference (src/kick_pme.cpp:20-29); the
        device mesh has no ghosts, so this only waits for the kick."""
        check(self.lib.tpm_synchronize(self.h), "kick_pme_end")

    def drift(self, dt: float) -> None:
        check(self.lib.tpm_drift(self.h, float(dt)), "drift")

    # ------------------------------------------------------- integration
    def integrate_begin(self, t0: float, scale: float = 1.0, first_call: bool = True) -> None:
        check(self.lib.tpm_integrate_begin(self.h, float(t0), float(scale), 1 if first_call else 0),
              "integrate_begin")

    def integrate_substep(self) -> dict:
        s = _lib.Substep()
        check(self.lib.tpm_integrate_substep(self.h, C.byref(s)), "integrate_substep")
        return {n: getattr(s, n) for n, _ in _lib.Substep._fields_}

    def integrate(self, t0: float, scale: float = 1.0, first_call: bool = True, max_substeps: int = 1 << 12):
        """One big step of rung-based kick-drift-kick; returns the substeps."""
        log = (_lib.Substep * max_substeps)()
        k = C.c_int()
        check(self.lib.tpm_integrate(self.h, float(t0), float(scale), 1 if first_call else 0, int(max_substeps),
                                     log, int(max_substeps), C.byref(k)), "integrate")
        return [{n: getattr(log[i], n) for n, _ in _lib.Substep._fields_} for i in range(k.value)]

    def diagnostics(self) -> dict:
        """FP64 per-particle kinetic and potential energy and momentum."""
        d = _lib.Diag()
        check(self.lib.tpm_diagnostics(self.h, C.byref(d)), "diagnostics")
        return {"kinetic": d.kinetic, "potential": d.potential, "momentum": list(d.momentum), "n": d.n}

    # ---------------------------------------------------------------- Ewald
    def gravity_short_ewald_call_kernel(self, sinkx, sinky, sinkz, method: int = 1):
        """FP64 Ewald at the sink positions from all particles of the box:
        returns (phi, (gx, gy, gz)) like src/gravity_short.cu:10-91."""
        sx = np.ascontiguousarray(sinkx, np.uint32)
        sy = np.ascontiguousarray(sinky, np.uint32)
        sz = np.ascontiguousarray(sinkz, np.uint32)
        ns = sx.size
        phi = np.empty(ns)
        g = [np.empty(ns) for _ in range(3)]
        check(self.lib.tpm_gravity_short_ewald(self.h, ns, _ptr(sx), _ptr(sy), _ptr(sz), int(method), _ptr(phi),
                                               *[_ptr(a) for a in g]), "gravity_short_ewald")
        return phi, tuple(g)

    def ewald_samples(self, idx: np.ndarray, method: int = 1):
        idx = np.ascontiguousarray(idx, np.int64)
        ns = idx.size
        phi = np.empty(ns)
        g = [np.empty(ns) for _ in range(3)]
        check(self.lib.tpm_ewald_fp64(self.h, ns, _ptr(idx), int(method), _ptr(phi), *[_ptr(a) for a in g]),
              "ewald_fp64")
        return phi, np.stack(g, axis=1)

    def gravity_short_ewald_compare(self, nsamples: int, seed: int = 1, method: int = 1) -> dict:
        """Errors of the last kick's forces against the FP64 Ewald sum on
        nsamples distinct particles (src/gravity_short.cpp:35-82)."""
        from .workloads import sample_indices
        idx = sample_indices(self.n, nsamples, seed)
        gx, gy, gz, pot = self.get_forces()
        phi, g = self.ewald_samples(idx, method)
        gk = np.stack([gx[idx], gy[idx], gz[idx]], axis=1)
        out = force_errors(gk, g, pot[idx], phi)
        out["samples"] = int(idx.size)
        return out

    # -------------------------------------------------------------- metrics
    def stage_times(self) -> dict:
        t = _lib.StageTimes()
        check(self.lib.tpm_get_stage_times(self.h, C.byref(t)), "get_stage_times")
        return {n: float(getattr(t, n)) for n, _ in _lib.StageTimes._fields_}

    def reset_stage_times(self) -> None:
        check(self.lib.tpm_reset_stage_times(self.h), "reset_stage_times")

    def launch_count(self) -> int:
        v = C.c_int64()
        check(self.lib.tpm_get_launch_count(self.h, C.byref(v)), "get_launch_count")
        return int(v.value)

    def device_bytes(self) -> int:
        v = C.c_int64()
        check(self.lib.tpm_ctx_device_bytes(self.h, C.byref(v)), "ctx_device_bytes")
        return int(v.value)

    def synchronize(self) -> None:
        check(self.lib.tpm_synchronize(self.h), "synchronize")

    def stream(self) -> int:
        p = C.c_void_p()
        check(self.lib.tpm_ctx_stream(self.h, C.byref(p)), "ctx_stream")
        return int(p.value or 0)

    def pme_step(self, min_rung: int = 0, scale: float = 1.0, t0: float = 1.0, first_call: bool = True) -> None:
        """chainmesh_create + gravity_long_compute(PME) + kick_pme, no host sync."""
        check(self.lib.tpm_pme_step(self.h, int(min_rung), float(scale), float(t0), 1 if first_call else 0),
              "pme_step")

    def pme_steps_host(self, inputs, outputs, min_rung: int = 0, scale: float = 1.0, t0: float = 1.0,
                       first_call: bool = True) -> None:
        """Served stream: one whole PME step per input particle set, host to
        host, transfers overlapped with the neighbouring steps' kernels.
        inputs / outputs: sequences of objects with x, y, z, vx, vy, vz, rung
        arrays (outputs may repeat one set).  Arrays must be C-contiguous and
        stay alive for the call."""
        ns = len(inputs)
        if len(outputs) != ns:
            raise ValueError("one output set per input set")
        n = int(inputs[0].x.size) if ns else 0
        def hp(p):
            return _lib.HostParticles(*[a.ctypes.data if hasattr(a, "ctypes") else int(a) for a in
                                        (p.x, p.y, p.z, p.vx, p.vy, p.vz, p.rung)])
        ins = (_lib.HostParticles * max(ns, 1))(*[hp(p) for p in inputs])
        outs = (_lib.HostParticles * max(ns, 1))(*[hp(p) for p in outputs])
        check(self.lib.tpm_pme_steps_host(self.h, ns, n, ins, outs, int(min_rung), float(scale), float(t0),
                                          1 if first_call else 0), "pme_steps_host")
        self.n = n

    def check_errors(self) -> None:
        check(self.lib.tpm_check_errors(self.h), "check_errors")

    def count_pairs(self, min_rung: int = 0):
        a = C.c_int64()
        b = C.c_int64()
        check(self.lib.tpm_count_pairs(self.h, int(min_rung), C.byref(a), C.byref(b)), "count_pairs")
        return int(a.value), int(b.value)


def ic_zeldovich(ctx: "TigerPM", n_side: int, seed: int, table_k=None, table_p=None, index: float = -2.0,
                 kcut_over_nyq: float = 0.5, rms_disp: float = 0.0) -> float:
    """Zel'dovich initial conditions generated on the device into ctx
    (tpm_ic_zeldovich): a power.init-style table (k h/Mpc, P (Mpc/h)^3) with
    the reference's sigma8 / growth-factor amplitude, or (no table)
    P ~ k^index exp(-k / (kcut_over_nyq k_Nyq)); rms_disp > 0 rescales to
    that rms displacement in particle spacings.  Returns max |dx| in spacings."""
    lib = _lib.load()
    p = _lib.ICParams()
    p.n_side = int(n_side)
    p.seed = int(seed)
    keep = []
    if table_k is not None:
        tk = np.ascontiguousarray(table_k, np.float64)
        tp = np.ascontiguousarray(table_p, np.float64)
        keep += [tk, tp]
        p.npower = tk.size
        p.power_k = tk.ctypes.data
        p.power_p = tp.ctypes.data
    p.index = float(index)
    p.kcut_over_nyq = float(kcut_over_nyq)
    p.rms_disp = float(rms_disp)
    dmax = C.c_double()
    check(lib.tpm_ic_zeldovich(ctx.h, C.byref(p), C.byref(dmax)), "ic_zeldovich")
    ctx.n = int(n_side) ** 3
    return float(dmax.value)


class Batch:
    """An ensemble of independent periodic boxes kicked together
    (tpm_batch_*): every box's sort and long-range solve run concurrently,
    then one interpolation launch and ONE persistent PP + kick launch over a
    (box, chain cell) work queue, optionally captured as a CUDA graph."""

    def __init__(self, opts_list, capacities):
        self.lib = _lib.load()
        nb = len(opts_list)
        if nb == 0 or len(capacities) != nb:
            raise ValueError("one capacity per box")
        self.opts = list(opts_list)
        arr = (Options * nb)(*opts_list)
        caps = (C.c_int64 * nb)(*[int(c) for c in capacities])
        h = C.c_void_p()
        check(self.lib.tpm_batch_create(nb, arr, caps, C.byref(h)), "batch_create")
        self.h = h
        self.nbox = nb
        self.counts = [0] * nb

    def close(self):
        if self.h:
            self.lib.tpm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_input(self, i: int, ps) -> None:
        x, y, z, vx, vy, vz, r = (np.ascontiguousarray(a) for a in
                                  (ps.x, ps.y, ps.z, ps.vx, ps.vy, ps.vz, ps.rung))
        check(self.lib.tpm_batch_set_input(self.h, int(i), x.size, _ptr(x), _ptr(y), _ptr(z), _ptr(vx), _ptr(vy),
                                           _ptr(vz), _ptr(r)), "batch_set_input")
        self.counts[i] = int(x.size)

    def box(self, i: int) -> TigerPM:
        """The context of box i (owned by the batch)."""
        h = C.c_void_p()
        check(self.lib.tpm_batch_box(self.h, int(i), C.byref(h)), "batch_box")
        return TigerPM.borrow(h, self.opts[i], self.counts[i])

    def step(self, restore: bool = True, graph: bool = True, min_rung: int = 0, scale: float = 1.0,
             t0: float = 1.0, first_call: bool = True) -> None:
        flags = (_lib.BATCH_RESTORE if restore else 0) | (_lib.BATCH_GRAPH if graph else 0)
        check(self.lib.tpm_batch_step(self.h, flags, int(min_rung), float(scale), float(t0),
                                      1 if first_call else 0), "batch_step")

    def steps_sequential(self, restore: bool = True, min_rung: int = 0, scale: float = 1.0, t0: float = 1.0,
                         first_call: bool = True) -> None:
        check(self.lib.tpm_batch_steps_sequential(self.h, 1 if restore else 0, int(min_rung), float(scale),
                                                  float(t0), 1 if first_call else 0), "batch_steps_sequential")

    def synchronize(self) -> None:
        check(self.lib.tpm_batch_synchronize(self.h), "batch_synchronize")

    def stream(self) -> int:
        p = C.c_void_p()
        check(self.lib.tpm_batch_stream(self.h, C.byref(p)), "batch_stream")
        return int(p.value or 0)

    def launch_count(self) -> int:
        v = C.c_int64()
        check(self.lib.tpm_batch_launch_count(self.h, C.byref(v)), "batch_launch_count")
        return int(v.value)

    def phase_times(self) -> dict:
        t = _lib.BatchTimes()
        check(self.lib.tpm_batch_phase_times(self.h, C.byref(t)), "batch_phase_times")
        return {n: float(getattr(t, n)) for n, _ in _lib.BatchTimes._fields_}

    def shape(self) -> dict:
        k = _lib.KickShape()
        check(self.lib.tpm_batch_get_shape(self.h, C.byref(k)), "batch_get_shape")
        return {n: getattr(k, n) for n, _ in _lib.KickShape._fields_}

    def set_shape(self, warps: int, stage: int, npass: int) -> None:
        k = _lib.KickShape(warps, stage, npass, 0, 0.0)
        check(self.lib.tpm_batch_set_shape(self.h, C.byref(k)), "batch_set_shape")

    def autotune(self, min_rung: int = 0, repeats: int = 2) -> dict:
        k = _lib.KickShape()
        check(self.lib.tpm_batch_autotune(self.h, int(min_rung), int(repeats), C.byref(k)), "batch_autotune")
        return {n: getattr(k, n) for n, _ in _lib.KickShape._fields_}


class Server:
    """A request loop serving kick + drift steps of resident boxes
    (tpm_serve_*): boxes are admitted against an HBM budget, requests start
    as slots and memory free up, and steps of different boxes overlap on the
    device."""

    def __init__(self, budget_bytes: int = 0, max_slots: int = 4):
        self.lib = _lib.load()
        h = C.c_void_p()
        check(self.lib.tpm_serve_create(int(budget_bytes), int(max_slots), C.byref(h)), "serve_create")
        self.h = h
        self.opts = []
        self.counts = []

    def close(self):
        if self.h:
            self.lib.tpm_serve_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add_box(self, opts: Options, ps) -> int:
        x, y, z, vx, vy, vz, r = (np.ascontiguousarray(a) for a in
                                  (ps.x, ps.y, ps.z, ps.vx, ps.vy, ps.vz, ps.rung))
        bid = C.c_int()
        check(self.lib.tpm_serve_add_box(self.h, C.byref(opts), x.size, _ptr(x), _ptr(y), _ptr(z), _ptr(vx),
                                         _ptr(vy), _ptr(vz), _ptr(r), C.byref(bid)), "serve_add_box")
        self.opts.append(opts)
        self.counts.append(int(x.size))
        return int(bid.value)

    def add_box_ic(self, opts: Options, n_side: int, seed: int, rms_disp: float = 0.3, index: float = -2.0,
                   kcut_over_nyq: float = 0.5) -> int:
        """Admits a box whose Zel'dovich particles are generated on the device
        (P ~ k^index exp(-k / (kcut k_Nyq)), rms displacement rms_disp spacings)."""
        p = _lib.ICParams()
        p.n_side = int(n_side)
        p.seed = int(seed)
        p.npower = 0
        p.index = float(index)
        p.kcut_over_nyq = float(kcut_over_nyq)
        p.rms_disp = float(rms_disp)
        bid = C.c_int()
        check(self.lib.tpm_serve_add_box_ic(self.h, C.byref(opts), C.byref(p), C.byref(bid)), "serve_add_box_ic")
        self.opts.append(opts)
        self.counts.append(int(n_side) ** 3)
        return int(bid.value)

    def submit(self, box: int, dt: float, min_rung: int = 0, scale: float = 1.0, t0: float = 1.0,
               first_call: bool = True) -> int:
        rid = C.c_int()
        check(self.lib.tpm_serve_submit(self.h, int(box), float(dt), int(min_rung), float(scale), float(t0),
                                        1 if first_call else 0, C.byref(rid)), "serve_submit")
        return int(rid.value)

    @staticmethod
    def _result(r) -> dict:
        return {n: getattr(r, n) for n, _ in _lib.ServeResult._fields_}

    def wait(self, req: int) -> dict:
        r = _lib.ServeResult()
        check(self.lib.tpm_serve_wait(self.h, int(req), C.byref(r)), "serve_wait")
        return self._result(r)

    def drain(self) -> None:
        check(self.lib.tpm_serve_drain(self.h), "serve_drain")

    def replay(self, boxes, arrivals_s, dt: float, min_rung: int = 0, scale: float = 1.0, t0: float = 1.0,
               first_call: bool = True):
        """Request i for boxes[i] submitted arrivals_s[i] seconds after the
        call starts; returns one result dict per request."""
        b = np.ascontiguousarray(boxes, np.int32)
        a = np.ascontiguousarray(arrivals_s, np.float64)
        res = (_lib.ServeResult * max(b.size, 1))()
        check(self.lib.tpm_serve_replay(self.h, int(b.size), _ptr(b), _ptr(a), float(dt), int(min_rung),
                                        float(scale), float(t0), 1 if first_call else 0, res), "serve_replay")
        return [self._result(res[i]) for i in range(b.size)]

    def box(self, i: int) -> TigerPM:
        """The context of an idle box (particles, chain-mesh offsets)."""
        h = C.c_void_p()
        check(self.lib.tpm_serve_box(self.h, int(i), C.byref(h)), "serve_box")
        return TigerPM.borrow(h, self.opts[i], self.counts[i])

    def stats(self) -> dict:
        s = _lib.ServeStats()
        check(self.lib.tpm_serve_stats(self.h, C.byref(s)), "serve_stats")
        return {n: getattr(s, n) for n, _ in _lib.ServeStats._fields_}


def fp32_peak_probe() -> float:
    """Measured FP32 FMA throughput of the current device, TFLOP/s."""
    lib = _lib.load()
    v = C.c_double()
    check(lib.tpm_fp32_peak_probe(C.byref(v)), "fp32_peak_probe")
    return float(v.value)
