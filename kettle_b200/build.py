"""Build the engine's shared libraries in-tree.

    python -m kettle_b200.build           # libkettle_b200.so (CUDA, sm_100a)

The CUDA library is compiled with nvcc for sm_100a only
(`-gencode arch=compute_100a,code=sm_100a`) and the CUDA runtime linked
statically, so the .so that travels with the repository needs nothing but the
driver.  Objects go to kettle_b200/_build/, the library to kettle_b200/lib/.
The C++20 drop-in front end (namespace ket) is built by `build_front_end()`.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = PKG / "host"
BUILD = PKG / "_build"
LIB = PKG / "lib"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"]

LIB_NAME = "libkettle_b200.so"
FRONT_NAME = "libket_b200.so"


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build kettle_b200")
    return cand


def _run(cmd: list[str]) -> str:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"command failed ({proc.returncode}): {' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
    return proc.stdout + proc.stderr


def _stale(out: pathlib.Path, deps: list[pathlib.Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


# headers the run-time compiled block kernels include (kt_jit.cpp embeds their text)
JIT_HEADERS = ("kt_complex.cuh", "kt_fused_dev.cuh", "kt_tma_dev.cuh")


def write_jit_headers() -> pathlib.Path:
    """BUILD/kt_jit_headers.inc: the text of JIT_HEADERS as C++ raw strings."""
    out = BUILD / "kt_jit_headers.inc"
    parts = ["// generated by kettle_b200/build.py from kettle_b200/csrc: do not edit",
             f"#define KT_JIT_N_HEADERS {len(JIT_HEADERS)}",
             "static const char* const KT_JIT_HEADER_NAMES[] = {" + ", ".join(f'"{h}"' for h in JIT_HEADERS) + "};",
             "static const char* const KT_JIT_HEADER_TEXT[] = {"]
    for h in JIT_HEADERS:
        text = (CSRC / h).read_text()
        if ")KTJIT\"" in text:
            raise RuntimeError(f"{h} contains the raw-string delimiter")
        parts.append('R"KTJIT(' + text + ')KTJIT",')
    parts.append("};")
    content = "\n".join(parts) + "\n"
    if not out.exists() or out.read_text() != content:
        out.write_text(content)
    return out


def build_library(verbose: bool = False, force: bool = False) -> pathlib.Path:
    """Compile every .cu/.cpp under csrc/ for sm_100a and link libkettle_b200.so."""
    BUILD.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    write_jit_headers()
    headers = sorted(CSRC.glob("*.cuh")) + [INCLUDE / "kettle_b200.h"]
    sources = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    jobs = []
    objs = []
    for src in sources:
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [nvcc(), *ARCH, *NVCC_FLAGS, f"-I{INCLUDE}", f"-I{CSRC}", f"-I{BUILD}", "-c", str(src), "-o", str(obj)]
            jobs.append(cmd)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    lib = LIB / LIB_NAME
    if force or jobs or _stale(lib, objs):
        _run([nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(lib), *map(str, objs), "-ldl"])
    return lib


def build_front_end(verbose: bool = False, force: bool = False) -> pathlib.Path:
    """Compile the C++20 `ket::` front end (host code over the C-ABI) into libket_b200.so."""
    lib = build_library(verbose=verbose, force=force)
    sources = sorted(HOST.glob("*.cpp"))
    if not sources:
        return lib
    headers = sorted((INCLUDE / "kettle").rglob("*.hpp")) + [INCLUDE / "kettle_b200.h"]
    out = LIB / FRONT_NAME
    if force or _stale(out, sources + headers + [lib]):
        cxx = shutil.which("g++") or "g++"
        cmd = [cxx, "-std=c++20", "-O2", "-fPIC", "-shared", f"-I{INCLUDE}", *map(str, sources),
               f"-L{LIB}", "-lkettle_b200", f"-Wl,-rpath,$ORIGIN", "-o", str(out)]
        text = _run(cmd)
        if verbose and text.strip():
            print(text)
    # the drop-in demonstration programs against this front end
    for src_name, exe_name in (("dropin_main.cpp", "dropin_b200"), ("dropin_host_main.cpp", "dropin_host_b200")):
        demo_src = ROOT / "tests" / "cpp" / src_name
        demo = LIB / exe_name
        if demo_src.exists() and (force or _stale(demo, [demo_src, out] + headers)):
            cxx = shutil.which("g++") or "g++"
            _run([cxx, "-std=c++20", "-O2", "-ffp-contract=off", f"-I{INCLUDE}", str(demo_src), f"-L{LIB}", "-lket_b200",
                  "-lkettle_b200", "-Wl,-rpath,$ORIGIN", "-o", str(demo)])
    return out


def build_oracle(verbose: bool = False) -> None:
    """Compile the oracle (test infrastructure): the C restatement always, and the
    reference library from its sources when they are present on this machine."""
    make = shutil.which("make") or "make"
    _run([make, "-C", str(ROOT / "oracle"), "port"])
    # oracle/Makefile knows where the kettle sources lie (KETTLE_REFERENCE
    # overrides it) and builds the reference only when they are there
    extra = [f"REF={os.environ['KETTLE_REFERENCE']}"] if os.environ.get("KETTLE_REFERENCE") else []
    _run([make, "-C", str(ROOT / "oracle"), "ref-if-present", *extra, f"-j{min(8, os.cpu_count() or 4)}"])


def ptxas_report() -> str:
    """Registers / spills / shared memory per kernel (nvcc -Xptxas -v)."""
    lines = []
    for src in sorted(CSRC.glob("*.cu")):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-Xptxas", "-v", f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(src),
               "-o", os.devnull]
        lines.append(_run(cmd))
    return "\n".join(lines)


if __name__ == "__main__":
    force = "--force" in sys.argv
    if "--ptxas" in sys.argv:
        print(ptxas_report())
        sys.exit(0)
    print(build_library(verbose=True, force=force))
    print(build_front_end(verbose=True, force=force))
