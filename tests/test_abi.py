"""CPU checks of the C ABI: the library loads, exports every entry point
declared in include/tpm.h, and the host-only option logic behaves like the
reference's process_options (src/options.cpp:37-118)."""
import ctypes as C
import math
import os
import re

import pytest

from tigerpm_b200 import _lib
from tigerpm_b200.api import make_options, options_for, process_options

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", f)).read()
            names |= set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(tpm_\w+)\s*\(", src, re.M))
    return names


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    bound = {s[0] for s in _lib.SIGNATURES}
    assert names <= bound | {"tpm_last_error_message"}


def test_options_derived_like_process_options():
    o = options_for(60, 3, 5)
    assert (o.four_dim, o.chain_dim, o.parts_o_chain) == (20, 4, 15)
    assert math.isclose(o.rs, 1 / 20) and o.GM == 1.0
    assert math.isclose(o.hsoft, 2 / 25 / 60) and math.isclose(o.eta, 0.2 / math.sqrt(2))
    assert math.isclose(o.code_to_cm, 7.108e26 * 60 / 1024 / 0.7)


def test_options_reject_where_reference_aborts():
    with pytest.raises(_lib.TPMError) as e:
        options_for(130, 3, 5)  # the reference's default: 130 % 15 != 0 -> abort()
    assert "multiple of 15" in str(e.value)


def test_options_parse_flags():
    o = process_options(["--parts_dim=64", "--four_dim", "64", "--chain_dim=11", "--rs_cells=1.25",
                         "--rcut_over_rs=4.5", "--assign=tsc", "--sort=fast", "--test=kick_pme"])
    assert (o.parts_dim, o.four_dim, o.chain_dim, o.assign, o.sort_mode) == (64, 64, 11, 2, 1)
    assert math.isclose(o.rs, 1.25 / 64) and o.rcut_over_rs == 4.5
    with pytest.raises(_lib.TPMError):
        process_options(["--no_such_flag=1"])
    with pytest.raises(_lib.TPMError):
        process_options(["--assign=ngp"])


def test_deposit_accumulator_option():
    """deterministic_deposit selects the deposit accumulator: 0 FP32 atomics
    (default), 1 exact int64, 2 26-bit fixed point; the header's constants
    match."""
    assert process_options(["--parts_dim=64", "--four_dim=64"]).deterministic_deposit == 0
    for v in (0, 1, 2):
        o = process_options(["--parts_dim=64", "--four_dim=64", f"--deterministic_deposit={v}"])
        assert o.deterministic_deposit == v
        assert make_options(16, 32, deterministic_deposit=v).deterministic_deposit == v
    assert make_options(16, 32, deterministic_deposit=True).deterministic_deposit == 1
    text = open(os.path.join(ROOT, "include", "tpm.h")).read()
    for name, v in (("TPM_DEPOSIT_FP32", 0), ("TPM_DEPOSIT_EXACT64", 1), ("TPM_DEPOSIT_FIXED32", 2)):
        assert re.search(rf"#define {name} {v}\b", text), name


def test_error_strings(lib):
    assert lib.tpm_error_string(0) == b"ok"
    assert b"rung" in lib.tpm_error_string(-6)
