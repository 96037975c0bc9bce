"""The allocation-free expectation entry point, kt_sv_expect_noalloc.

It serves callers that cannot let the library allocate device memory (a host
that owns every byte through its own pool, a loop that must not allocate
while running): its scratch is a fixed array inside the library.  Called
through the C-ABI on a raw device pointer, it must give the values of the
allocating kt_sv_expect within 1e-12, on two calls in a row (the second call
reuses the array the first one left behind), and reject operators larger
than its fixed capacity.

This file is named to be collected last, so a run that stops at its first
failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import random_state
from kettle_b200 import capi
from kettle_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _noalloc(sv: capi.Statevector, strings, coeffs):
    n = C.c_int32()
    dt = C.c_int32()
    ptr = C.c_void_p()
    capi.check(capi.lib().kt_sv_info(sv.handle, C.byref(n), C.byref(dt), C.byref(ptr)))
    s = np.ascontiguousarray(strings, dtype=capi.PAULI_DTYPE)
    c = np.ascontiguousarray(coeffs, dtype=np.complex128)
    terms = np.empty(s.size, dtype=np.complex128)
    total = np.empty(1, dtype=np.complex128)
    capi.check(capi.lib().kt_sv_expect_noalloc(ptr, n.value, dt.value, capi.ptr(s), s.size, capi.ptr(c),
                                               capi.ptr(terms), capi.ptr(total), None))
    return terms, complex(total[0])


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
    sv.close()


def test_noalloc_rejects_oversized_operator(engine):
    sv = capi.Statevector(6)
    strings, coeffs = W.random_paulis(6, 513, 3)
    with pytest.raises(capi.KettleError) as e:
        _noalloc(sv, strings, coeffs)
    assert "at most 512" in str(e.value)
    sv.close()
