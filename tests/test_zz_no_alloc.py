"""The allocation-free expectation entry point, kt_sv_expect_noalloc.

It serves callers that cannot let the library allocate device memory (a host
that owns every byte through its own pool, a loop that must not allocate
while running): its scratch is a fixed array inside the library.  Called
through the C-ABI on a raw device pointer, it must give the values of the
allocating kt_sv_expect (bit for bit on a GPU of up to 148 SMs, within 1e-12
on any), on two calls in a row (the second call reuses the array the first
one left behind), on the default stream and on a stream the caller created;
it must allocate no device memory, and reject operators larger than its
fixed capacity.

This file is named to be collected last, so a run that stops at its first
failure has run every other test before it.
"""
import ctypes as C
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from conftest import ROOT, random_state
from kettle_b200 import capi
from kettle_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _noalloc(sv: capi.Statevector, strings, coeffs, stream=None):
    n = C.c_int32()
    dt = C.c_int32()
    ptr = C.c_void_p()
    capi.check(capi.lib().kt_sv_info(sv.handle, C.byref(n), C.byref(dt), C.byref(ptr)))
    s = np.ascontiguousarray(strings, dtype=capi.PAULI_DTYPE)
    c = np.ascontiguousarray(coeffs, dtype=np.complex128)
    terms = np.empty(s.size, dtype=np.complex128)
    total = np.empty(1, dtype=np.complex128)
    capi.check(capi.lib().kt_sv_expect_noalloc(ptr, n.value, dt.value, capi.ptr(s), s.size, capi.ptr(c),
                                               capi.ptr(terms), capi.ptr(total), stream))
    return terms, complex(total[0])


def _small_gpu():
    import torch
    return torch.cuda.get_device_properties(0).multi_processor_count <= 148


@pytest.mark.parametrize("n,dtype", [(11, capi.KT_C128), (20, capi.KT_C128), (16, capi.KT_C64)])
def test_noalloc_matches_allocating_path_twice(engine, n, dtype):
    sv = capi.Statevector(n, dtype)
    sv.upload(random_state(n, n))
    for call, (count, seed) in enumerate(((300, 1), (120, 2))):
        strings, coeffs = W.random_paulis(n, count, seed + 10 * n)
        want_terms, want_total = sv.expect(strings, coeffs)
        got_terms, got_total = _noalloc(sv, strings, coeffs)
        assert np.abs(got_terms - want_terms).max() < TOL, call
        assert abs(got_total - want_total) < TOL, call
        if _small_gpu():
            assert np.array_equal(got_terms, want_terms), call
            assert got_total == want_total, call
    sv.close()


def test_noalloc_on_a_caller_stream(engine):
    """The same values when the caller passes a stream of its own; the state is
    written on that stream just before the call, so the call must be ordered
    after it."""
    import torch
    n = 18
    st = torch.cuda.Stream()
    sv = capi.Statevector(n, stream=st.cuda_stream)
    strings, coeffs = W.random_paulis(n, 200, 5)
    for k in range(2):
        sv.set_basis(k)
        sv.apply(W.random_layers(n, 3, seed=60 + k, mixed=True))
        got_terms, got_total = _noalloc(sv, strings, coeffs, stream=C.c_void_p(st.cuda_stream))
        want_terms, want_total = sv.expect(strings, coeffs)
        assert np.abs(got_terms - want_terms).max() < TOL, k
        assert abs(got_total - want_total) < TOL, k
    sv.close()


_ALLOC_PROBE = textwrap.dedent(r"""
    import ctypes as C, glob, json, os, sys
    import numpy as np
    sys.path.insert(0, sys.argv[1])
    from kettle_b200 import capi
    from kettle_b200 import workloads as W
    # the CUDA runtime as a shared library, for cudaMemGetInfo on the same
    # (primary) context the engine uses; torch is not loaded
    cands = glob.glob(os.path.join(sys.prefix, "lib", "python3*", "site-packages", "nvidia", "cuda_runtime", "lib",
                                   "libcudart.so.*")) + ["/usr/local/cuda/lib64/libcudart.so.12", "libcudart.so.12"]
    rt = None
    for c in cands:
        try:
            rt = C.CDLL(c)
            break
        except OSError:
            continue
    assert rt is not None, "no CUDA runtime library"
    def free_bytes():
        assert rt.cudaDeviceSynchronize() == 0
        f, t = C.c_size_t(), C.c_size_t()
        assert rt.cudaMemGetInfo(C.byref(f), C.byref(t)) == 0
        return f.value
    n = 20
    sv = capi.Statevector(n)
    sv.set_basis(3)
    strings, coeffs = W.random_paulis(n, 400, 9)
    many, many_c = W.random_paulis(n, 1200, 10)
    nq, dt, ptr = C.c_int32(), C.c_int32(), C.c_void_p()
    capi.check(capi.lib().kt_sv_info(sv.handle, C.byref(nq), C.byref(dt), C.byref(ptr)))
    s = np.ascontiguousarray(strings, dtype=capi.PAULI_DTYPE)
    c = np.ascontiguousarray(coeffs, dtype=np.complex128)
    terms = np.empty(s.size, dtype=np.complex128)
    total = np.empty(1, dtype=np.complex128)
    free = [free_bytes()]
    for _ in range(2):
        capi.check(capi.lib().kt_sv_expect_noalloc(ptr, nq.value, dt.value, capi.ptr(s), s.size, capi.ptr(c),
                                                   capi.ptr(terms), capi.ptr(total), None))
        free.append(free_bytes())
    sv.expect(many, many_c)  # the allocating path grows the handle's scratch (~5.7 MB)
    free.append(free_bytes())
    print(json.dumps(free))
""")


def test_noalloc_allocates_no_device_memory(engine):
    """In a fresh process whose modules load eagerly (so the library's fixed
    array is in place before anything is measured; torch is not imported, so
    only the engine and the CUDA runtime load), the free device memory is
    the same before and after the first and second call; the allocating
    kt_sv_expect afterwards lowers it, which shows the measurement sees an
    allocation of this size."""
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    out = subprocess.run([sys.executable, "-c", _ALLOC_PROBE, str(ROOT)], capture_output=True, text=True,
                         env=env, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    free = [int(v) for v in out.stdout.strip().splitlines()[-1].strip("[]").split(",")]
    assert free[1] == free[0] and free[2] == free[0], free
    assert free[3] < free[0], free


def test_noalloc_rejects_oversized_operator(engine):
    sv = capi.Statevector(6)
    strings, coeffs = W.random_paulis(6, 513, 3)
    with pytest.raises(capi.KettleError) as e:
        _noalloc(sv, strings, coeffs)
    assert "at most 512" in str(e.value)
    sv.close()
