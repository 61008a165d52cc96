"""tpm_ewald_fp64_noalloc: the FP64 Ewald sum for callers that may not allocate
device memory (a host that owns all device memory through its own pool, or an
allocation-free hook inside a running step).  Its scratch is a fixed buffer
inside the library, so the test checks that two calls in a row -- the second
on different sinks, over whatever the first left in that buffer -- agree with
tpm_gravity_short_ewald (method 1), which uses freshly allocated scratch.

This file is collected last on purpose: a run that stops at the first failure
has run every other test before it."""
import ctypes as C
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from golden_io import load, names
from helpers import particle_set, rel_rms
from tigerpm_b200 import _lib
from tigerpm_b200 import workloads as W
from tigerpm_b200.api import TigerPM, make_options

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_noalloc_ewald_matches_allocating_path_twice():
    import torch
    lib = _lib.load()
    ps = particle_set("halos", 20, 41)
    opts = make_options(20, 20, rs_cells=1.0)
    ref = []
    sinks = []
    with TigerPM(opts, ps.n) as t:
        t.set_particles(ps)
        for seed in (3, 4):
            idx = W.sample_indices(ps.n, 96 if seed == 3 else 40, seed)
            sx, sy, sz = ps.x[idx].copy(), ps.y[idx].copy(), ps.z[idx].copy()
            sx[0] = sx[0] + 777  # a near pair that is not the sink itself
            phi, g = t.gravity_short_ewald_call_kernel(sx, sy, sz, method=1)
            ref.append((phi, np.stack(g, 1)))
            sinks.append((sx, sy, sz))
    x, y, z = (_dev(torch, a) for a in (ps.x, ps.y, ps.z))
    stream = torch.cuda.current_stream().cuda_stream
    for (sx, sy, sz), (rphi, rg) in zip(sinks, ref):
        ns = sx.size
        dsx, dsy, dsz = (_dev(torch, a) for a in (sx, sy, sz))
        out = [torch.full((ns,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(4)]
        rc = lib.tpm_ewald_fp64_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                        C.c_void_p(z.data_ptr()), ps.n, C.c_void_p(dsx.data_ptr()),
                                        C.c_void_p(dsy.data_ptr()), C.c_void_p(dsz.data_ptr()), ns, opts.hsoft,
                                        *[C.c_void_p(o.data_ptr()) for o in out], C.c_void_p(stream))
        _lib.check(rc, "tpm_ewald_fp64_noalloc")
        torch.cuda.synchronize()
        phi = out[0].cpu().numpy()
        g = torch.stack(out[1:], 1).cpu().numpy()
        assert np.all(np.isfinite(phi)) and np.all(np.isfinite(g))
        assert rel_rms(phi, rphi) < 1e-9
        assert rel_rms(g, rg) < 1e-9


def _call(lib, torch, src, n, snk, out, stream, hsoft):
    rc = lib.tpm_ewald_fp64_noalloc(*[C.c_void_p(a.data_ptr()) for a in src], n,
                                    *[C.c_void_p(a.data_ptr()) for a in snk], int(snk[0].numel()), hsoft,
                                    *[C.c_void_p(o.data_ptr()) for o in out], stream)
    _lib.check(rc, "tpm_ewald_fp64_noalloc")


def test_noalloc_ewald_allocates_nothing():
    """After a first call (which only looks up the library's buffer), further
    calls on other sinks leave the device's free memory and torch's allocator
    untouched."""
    import torch
    lib = _lib.load()
    ps = particle_set("uniform", 16, 43)
    src = [_dev(torch, a) for a in (ps.x, ps.y, ps.z)]
    snk = [_dev(torch, a[:64]) for a in (ps.x, ps.y, ps.z)]
    snk2 = [_dev(torch, a[100:131]) for a in (ps.x, ps.y, ps.z)]
    out = [torch.empty(64, dtype=torch.float64, device="cuda") for _ in range(4)]
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _call(lib, torch, src, ps.n, snk, out, stream, 0.01)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    stats0 = torch.cuda.memory_stats()
    for _ in range(3):
        _call(lib, torch, src, ps.n, snk2, [o[:31] for o in out], stream, 0.01)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    stats1 = torch.cuda.memory_stats()
    assert free1 == free0
    for k in ("allocation.all.allocated", "segment.all.allocated", "reserved_bytes.all.allocated"):
        assert stats1.get(k, 0) == stats0.get(k, 0), k


def test_noalloc_ewald_first_call_on_nonblocking_stream():
    """The very first call in a process, queued on a non-blocking stream,
    already sees the reciprocal-vector table its set-up copies."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = textwrap.dedent("""
        import ctypes as C, sys
        import numpy as np, torch
        sys.path.insert(0, %r); sys.path.insert(0, %r)
        from tigerpm_b200 import _lib
        from helpers import particle_set, rel_rms
        from tigerpm_b200.api import TigerPM, make_options
        lib = _lib.load()
        ps = particle_set("halos", 16, 47)
        sx, sy, sz = ps.x[:50].copy(), ps.y[:50].copy(), ps.z[:50].copy()
        s = torch.cuda.Stream()  # created with cudaStreamNonBlocking
        src = [torch.from_numpy(a).cuda() for a in (ps.x, ps.y, ps.z)]
        snk = [torch.from_numpy(a).cuda() for a in (sx, sy, sz)]
        out = [torch.empty(50, dtype=torch.float64, device="cuda") for _ in range(4)]
        torch.cuda.synchronize()
        rc = lib.tpm_ewald_fp64_noalloc(*[C.c_void_p(a.data_ptr()) for a in src], ps.n,
                                        *[C.c_void_p(a.data_ptr()) for a in snk], 50, 0.005,
                                        *[C.c_void_p(o.data_ptr()) for o in out], C.c_void_p(s.cuda_stream))
        _lib.check(rc, "noalloc")
        s.synchronize()
        opts = make_options(16, 16, rs_cells=1.0)
        opts.hsoft = 0.005
        with TigerPM(opts, ps.n) as t:
            t.set_particles(ps)
            phi, g = t.gravity_short_ewald_call_kernel(sx, sy, sz, method=1)
        assert rel_rms(out[0].cpu().numpy(), phi) < 1e-9
        assert rel_rms(torch.stack(out[1:], 1).cpu().numpy(), np.stack(g, 1)) < 1e-9
        print("ok")
    """) % (root, os.path.join(root, "tests"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr


def test_noalloc_ewald_rejects_too_many_sinks():
    lib = _lib.load()
    rc = lib.tpm_ewald_fp64_noalloc(None, None, None, 0, None, None, None, _lib.TPM_EWALD_NOALLOC_MAX_SINKS + 1,
                                    0.01, None, None, None, None, None)
    assert rc == _lib.TPM_ERR_INVALID
    assert b"exceed its maximum" in lib.tpm_last_error_message()


@pytest.mark.parametrize("case", names("ewald"))
def test_noalloc_ewald_matches_reference_golden(case):
    """Against the reference's own Ewald kernel (golden vectors)."""
    import torch
    d = load("ewald_" + case)
    s = d["sink_index"]
    src = [_dev(torch, d[k].view(np.int32)) for k in ("x", "y", "z")]
    snk = [_dev(torch, d[k][s].view(np.int32)) for k in ("x", "y", "z")]
    ns = int(s.size)
    out = [torch.empty(ns, dtype=torch.float64, device="cuda") for _ in range(4)]
    torch.cuda.synchronize()
    rc = _lib.load().tpm_ewald_fp64_noalloc(*[C.c_void_p(a.data_ptr()) for a in src], int(d["x"].size),
                                            *[C.c_void_p(a.data_ptr()) for a in snk], ns, float(d["hsoft"]),
                                            *[C.c_void_p(o.data_ptr()) for o in out], None)
    _lib.check(rc, "tpm_ewald_fp64_noalloc")
    torch.cuda.synchronize()
    phi, gx, gy, gz = (o.cpu().numpy() for o in out)
    assert rel_rms(np.stack([gx, gy, gz], 1), np.stack([d["gx"], d["gy"], d["gz"]], 1)) < 1e-5
    assert rel_rms(phi, d["phi"]) < 1e-5
