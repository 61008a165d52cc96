"""The reference's own C++ call sequence (kick_pme_test, src/test.cpp:182-234)
against include/tpm_reference.hpp, compiled and linked to the library."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "tigerpm_b200")
NVCC = "/usr/local/cuda/bin/nvcc"
REF = os.environ.get("REF", "/root/reference")  # the reference source tree, when mounted


def build_driver(tmp_path):
    exe = str(tmp_path / "ref_driver")
    subprocess.run([NVCC, "-std=c++17", "-O2", "-x", "cu", os.path.join(ROOT, "tests", "cpp", "ref_driver.cpp"),
                    "-I" + INC, "-L" + LIBDIR, "-ltigerpm_b200", "-Xlinker", "-rpath=" + LIBDIR, "-o", exe],
                   check=True)
    return exe


def test_driver_compiles(tmp_path):
    """The reference-signature header and the driver compile and link (CPU)."""
    assert os.path.exists(build_driver(tmp_path))


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not mounted")
def test_shim_matches_reference_headers(tmp_path):
    """reference_api.cpp type-checks against the reference's own headers
    (TPM_REFERENCE_GLOBALS_EXTERNAL), i.e. it defines exactly the functions
    the reference declares."""
    out = str(tmp_path / "ref_api.o")
    subprocess.run([NVCC, "-std=c++17", "-x", "cu", "-c", os.path.join(ROOT, "tigerpm_b200", "csrc", "reference_api.cpp"),
                    "-DTPM_REFERENCE_GLOBALS_EXTERNAL", "-I" + REF, "-I" + INC, "-include", "string",
                    "-o", out], check=True)
    assert os.path.exists(out)


@pytest.mark.gpu
def test_kick_pme_test_sequence(tmp_path):
    exe = build_driver(tmp_path)
    r = subprocess.run([exe, "--parts_dim=48", "--four_dim=96", "--chain_dim=8", "--rs_cells=2.0",
                        "--rcut_over_rs=6.0"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    line = [l for l in r.stdout.splitlines() if l.startswith("RESULT")][0]
    kv = dict(t.split("=") for t in line.split()[1:])
    assert int(kv["cells_bad"]) == 0 and int(kv["misplaced"]) == 0
    assert int(kv["total"]) == 48 ** 3
    assert int(kv["phi_box"]) == (96 + 6) ** 3
    assert float(kv["force_rms_vector"]) < 2e-4, line
