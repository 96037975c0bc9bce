"""Drop-in check of kettle's host-side API: tests/cpp/dropin_host_main.cpp
uses only the kettle C++ API (bitstring / state-index / dynamic-bitset
conversions, binary fraction expansions, marginal strips, seeded random 2x2
unitaries and random states, state projections, n-local circuits, integer
ranges, circuit adders and compound gates with their range errors,
transpiled circuits, classical registers and control-flow predicates, 2x2
matrix arithmetic and square roots, Pauli strings and operators, readout
noise, memory-to-counts; and, holding states, random states, projections
and the io/ text formats).  Built against the reference
(oracle/_ref/dropin_host_ref, from the reference's own sources) and against
this engine's ket:: front end (kettle_b200/lib/dropin_host_b200), both must
print the same text; doubles are printed in hexadecimal, so equal text is
equal bits, and errors print the thrown message.

The state part holds its states in GPU memory on the front end: on the CPU it
runs over host-memory stand-ins of the six state calls of the C-ABI
(tests/cpp/fake_state_abi.c, preloaded), which checks the front end's host
logic; on a GPU it runs through the engine itself
(tests/test_gpu_state_utils.py)."""
import os
import pathlib
import shutil
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
REF_BIN = ROOT / "oracle" / "_ref" / "dropin_host_ref"
OUR_BIN = ROOT / "kettle_b200" / "lib" / "dropin_host_b200"


def _run(exe, mode, env=None):
    out = subprocess.run([str(exe), mode], capture_output=True, text=True, timeout=300, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    return out.stdout


def _ref(mode):
    if not REF_BIN.exists():
        pytest.skip("reference build of the host-utility program not present (oracle/_ref)")
    return _run(REF_BIN, mode)


def _diff(a, b):
    la, lb = a.splitlines(), b.splitlines()
    for k, (x, y) in enumerate(zip(la, lb)):
        if x != y:
            return f"line {k}: reference {x!r} != engine {y!r}"
    return f"{len(la)} lines against {len(lb)}"


def test_host_utilities_match_reference():
    want = _ref("host")
    assert OUR_BIN.exists(), "front-end build of the host-utility program missing (kettle_b200.build)"
    got = _run(OUR_BIN, "host")
    assert got == want, _diff(want, got)
    assert "useed 11" in got and "err rstrip" in got and got.count("\nconv ") == 61  # 2 + 4 + ... + 32 indices, less the first


def test_state_utilities_match_reference_on_host_state_calls(tmp_path):
    want = _ref("states")
    assert OUR_BIN.exists(), "front-end build of the host-utility program missing (kettle_b200.build)"
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler for the host-memory state calls")
    fake = tmp_path / "fake_state_abi.so"
    subprocess.run([cc, "-std=c11", "-O2", "-shared", "-fPIC", f"-I{ROOT / 'include'}",
                    str(ROOT / "tests" / "cpp" / "fake_state_abi.c"), "-o", str(fake)], check=True)
    env = dict(os.environ, LD_PRELOAD=str(fake))
    got = _run(OUR_BIN, "states", env=env)
    assert got == want, _diff(want, got)
    assert got.count("err project ") == 5 and "proj_basis 0 0 0x1p+0" in got
