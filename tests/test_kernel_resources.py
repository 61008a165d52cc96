"""The hot kernels compile for sm_100a without local memory: no stack frame
and no register spills.  A value that falls to local memory costs these
loops several percent (a float4 taken by reference in the kick's buffer
tail cost 6 % of the kick), so the property is checked on the CPU with
nvcc -Xptxas -v, with the library's own build flags."""
import concurrent.futures
import os
import re
import subprocess
import tempfile

import pytest

from tigerpm_b200 import build as B

# source file -> kernels (a regex on the mangled name) that must use neither
# a stack frame nor spills
HOT = {
    "kick_pme.cu": [r"k_kick_pme", r"k_kick_batch", r"k_kick_slots"],
    "gravity_long.cu": [r"k_deposit"],
    "fft3d.cu": [r"k_line_x_greenILi768E", r"k_line_z_r2cILi768E"],
}


def ptxas_report(src):
    """{mangled kernel name: (stack bytes, spill store bytes, spill load bytes)}"""
    with tempfile.TemporaryDirectory() as d:
        cmd = [B.nvcc()] + B.ARCH + B.NVCC_FLAGS + ["-Xptxas", "-v", "-c", os.path.join(B.CSRC, src),
                                                   "-o", os.path.join(d, "x.o")]
        out = subprocess.run(cmd, capture_output=True, text=True, check=True).stderr
    report, name = {}, None
    for line in out.splitlines():
        m = re.search(r"Compiling entry function '([^']+)'", line)
        if m:
            name = m.group(1)
            continue
        m = re.search(r"(\d+) bytes stack frame, (\d+) bytes spill stores, (\d+) bytes spill loads", line)
        if m and name:
            report[name] = tuple(int(g) for g in m.groups())
            name = None
    return report


def nvcc_available():
    try:
        B.nvcc()
        return True
    except RuntimeError:
        return False


@pytest.mark.skipif(not nvcc_available(), reason="nvcc not found")
def test_hot_kernels_use_no_local_memory():
    with concurrent.futures.ThreadPoolExecutor(len(HOT)) as ex:
        reports = dict(zip(HOT, ex.map(ptxas_report, HOT)))
    for src, patterns in HOT.items():
        for pat in patterns:
            hits = {k: v for k, v in reports[src].items() if re.search(pat, k)}
            assert hits, (src, pat)
            bad = {k: v for k, v in hits.items() if any(v)}
            assert not bad, (src, pat, bad)
