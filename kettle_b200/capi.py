"""ctypes binding of the engine's C-ABI (include/kettle_b200.h).

This is the Python face of the same entry points a C, C++ or Go caller binds.
Loading fails loudly when libkettle_b200.so is missing: there is no CPU
fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

LIB_PATH = pathlib.Path(__file__).resolve().parent / "lib" / "libkettle_b200.so"

KT_OK = 0
KT_ERR_INVALID = -1
KT_ERR_CUDA = -2
KT_ERR_NOMEM = -3
KT_ERR_QUBITS = -4
KT_ERR_TIMEOUT = -5
KT_ERR_UNSUPPORTED = -6
KT_C128 = 0
KT_C64 = 1
KT_APPLY_FUSED = 0
KT_APPLY_PER_GATE = 1

# ket::Gate numbering (include/kettle/gates/primitive_gate.hpp:19-52 of the reference)
GATES = ["H", "X", "Y", "Z", "S", "SDAG", "T", "TDAG", "SX", "SXDAG", "RX", "RY", "RZ", "P",
         "CH", "CX", "CY", "CZ", "CS", "CSDAG", "CT", "CTDAG", "CSX", "CSXDAG", "CRX", "CRY", "CRZ", "CP",
         "U", "CU", "M"]
OP = {name: i for i, name in enumerate(GATES)}
ANGLE_GATES = {"RX", "RY", "RZ", "P", "CRX", "CRY", "CRZ", "CP"}
CONTROLLED = {g for g in GATES if g.startswith("C") and g not in ("CU",)} | {"CU"}

# numpy mirrors of the C records
GATE_DTYPE = np.dtype([("op", "u1"), ("r0", "u1"), ("r1", "<u2"), ("target", "<u4"), ("control", "<u4"),
                       ("param", "<i4"), ("angle", "<f8"), ("u", "<f8", (8,))], align=True)
PAULI_DTYPE = np.dtype([("x", "<u8"), ("z", "<u8"), ("phase", "<i4"), ("r", "<i4")], align=True)
BATCH_ITEM_DTYPE = np.dtype([("n_qubits", "<i4"), ("r", "<i4"), ("gate_offset", "<i8"), ("n_gates", "<i8"),
                             ("param_offset", "<i8"), ("n_params", "<i8"), ("string_offset", "<i8"),
                             ("n_strings", "<i8")], align=True)
assert GATE_DTYPE.itemsize == 88 and PAULI_DTYPE.itemsize == 24 and BATCH_ITEM_DTYPE.itemsize == 56


class KettleError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


_lib = None

P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64
U32 = C.c_uint32
U64 = C.c_uint64
DP = C.POINTER(C.c_double)

_SIGS = {
    "kt_last_error": ([], C.c_char_p),
    "kt_version": ([], I32),
    "kt_device_synchronize": ([], I32),
    "kt_canonicals_mt19937": ([U32, I64, P], I32),
    "kt_tuning_set": ([C.c_char_p, I64], I32),
    "kt_tuning_get": ([C.c_char_p, C.POINTER(I64)], I32),
    "kt_jit_stats": ([P, P, P], I32),
    "kt_jit_cache_stats": ([P, P], I32),
    "kt_sv_prepare": ([P, P, I64, P, I64], I32),
    "kt_jit_compile_only": ([I32, I32, P, I64, P, I64, P], I32),
    "kt_sv_create": ([I32, I32, C.POINTER(P)], I32),
    "kt_sv_wrap": ([P, I32, I32, C.POINTER(P)], I32),
    "kt_sv_destroy": ([P], I32),
    "kt_sv_set_stream": ([P, P], I32),
    "kt_sv_info": ([P, C.POINTER(I32), C.POINTER(I32), C.POINTER(P)], I32),
    "kt_sv_set_basis": ([P, U64], I32),
    "kt_sv_upload": ([P, P, U64], I32),
    "kt_sv_download": ([P, P, U64], I32),
    "kt_sv_copy": ([P, P], I32),
    "kt_sv_apply": ([P, P, I64, P, I64, I32], I32),
    "kt_sv_apply_stats": ([P, C.POINTER(I64), DP], I32),
    "kt_dm_apply_stats": ([P, C.POINTER(I64), DP], I32),
    "kt_plan_blocks": ([I32, P, I64, P, I64, P, I64, C.POINTER(I64)], I32),
    "kt_sv_tensor_product": ([P, P, P], I32),
    "kt_sv_diagonal_expectation": ([P, P, P], I32),
    "kt_sv_apply_dense5": ([P, P, I32], I32),
    "kt_sample_probabilities": ([P, U64, P, I64, P, I32, P], I32),
    "kt_dm_measure_probs": ([P, U32, DP, DP], I32),
    "kt_dm_collapse": ([P, U32, I32, C.c_double], I32),
    "kt_plan_stats": ([I32, I32, P, I64, P, I64, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64), C.POINTER(I64)], I32),
    "kt_plan_order": ([I32, I32, P, I64, P, I64, P, I64, C.POINTER(I64)], I32),
    "kt_sv_expect": ([P, P, I64, P, P, P], I32),
    "kt_sv_expect_noalloc": ([P, I32, I32, P, I64, P, P, P, P], I32),
    "kt_sv_probabilities": ([P, P, P], I32),
    "kt_sv_sample": ([P, P, P, I64, P, I32, C.POINTER(I32)], I32),
    "kt_sv_measure_probs": ([P, U32, DP, DP], I32),
    "kt_sv_collapse": ([P, U32, I32, C.c_double], I32),
    "kt_sv_norm_sq": ([P, DP], I32),
    "kt_sv_inner": ([P, P, P], I32),
    "kt_pairs_single": ([U32, U32, U64, U64, P], I32),
    "kt_pairs_double": ([U32, U32, U32, I32, U64, U64, P], I32),
    "kt_dm_create": ([I32, I32, C.POINTER(P)], I32),
    "kt_dm_destroy": ([P], I32),
    "kt_dm_set_stream": ([P, P], I32),
    "kt_dm_set_basis": ([P, U64], I32),
    "kt_dm_upload": ([P, P, U64], I32),
    "kt_dm_download": ([P, P, U64], I32),
    "kt_dm_apply": ([P, P, I64, P, I64, I32], I32),
    "kt_dm_prepare": ([P, P, I64, P, I64], I32),
    "kt_dm_expect": ([P, P, I64, P, P, P], I32),
    "kt_dm_trace": ([P, P], I32),
    "kt_dm_probabilities": ([P, P], I32),
    "kt_dm_partial_trace": ([P, P, I32, P], I32),
    "kt_dm_tensor_product": ([P, P, P], I32),
    "kt_dm_trace_of_square": ([P, P], I32),
    "kt_adjoint_create": ([P, I32, C.POINTER(P)], I32),
    "kt_adjoint_destroy": ([P], I32),
    "kt_adjoint_forward": ([P, P, I64, P, I64, P, I64, P, DP], I32),
    "kt_adjoint_backward": ([P, P, I64], I32),
    "kt_batch_create": ([P, I64, P, I64, I64, P, P, I64, I32, I32, C.POINTER(P)], I32),
    "kt_batch_set_stream": ([P, P], I32),
    "kt_batch_evaluate": ([P, P, P, P], I32),
    "kt_batch_stats": ([P] + [C.POINTER(I64)] * 6 + [DP, DP], I32),
    "kt_batch_compiled": ([P, C.POINTER(I64), C.POINTER(I64)], I32),
    "kt_batch_destroy": ([P], I32),
    "kt_batch_run": ([P, I64, P, I64, P, I64, P, P, I64, I32, P, P, P], I32),
}


def lib() -> C.CDLL:
    """Load libkettle_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m kettle_b200.build` "
                               "(the engine has no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


def check(rc: int) -> None:
    if rc != KT_OK:
        msg = lib().kt_last_error().decode(errors="replace")
        raise KettleError(rc, msg)


def ptr(a) -> int | None:
    """Data pointer of a numpy array (None for None)."""
    if a is None:
        return None
    return a.ctypes.data


def canonicals_mt19937(seed: int, n: int) -> np.ndarray:
    """std::generate_canonical<double,53>(std::mt19937(seed)) draws, from the library's host code."""
    out = np.empty(n, dtype=np.float64)
    check(lib().kt_canonicals_mt19937(seed & 0xFFFFFFFF, n, ptr(out)))
    return out


def plan_stats(n_qubits: int, gates: np.ndarray, params: np.ndarray | None = None, dtype: int = KT_C128) -> dict:
    """Host-only dry run of the fused planner (no GPU needed)."""
    g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
    p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
    out = [I64(0) for _ in range(4)]
    check(lib().kt_plan_stats(n_qubits, dtype, ptr(g), g.size, ptr(p), 0 if p is None else p.size,
                              *[C.byref(o) for o in out]))
    return dict(zip(("blocks", "phases", "ops", "transposes"), (int(o.value) for o in out)))


def plan_order(n_qubits: int, gates: np.ndarray, params: np.ndarray | None = None, dtype: int = KT_C128) -> np.ndarray:
    """Host-only: the fused planner's gates (lowered-stream indices) in the order they take effect."""
    g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
    p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
    out = np.zeros(max(1, 2 * g.size), dtype=np.int64)
    cnt = I64(0)
    check(lib().kt_plan_order(n_qubits, dtype, ptr(g), g.size, ptr(p), 0 if p is None else p.size,
                              ptr(out), out.size, C.byref(cnt)))
    return out[:cnt.value].copy()


def plan_blocks(n_qubits: int, gates: np.ndarray, params: np.ndarray | None = None) -> np.ndarray:
    """Per fused block of a complex128 apply: [ops, phases, transposes, FP64 per amplitude] (kt_plan_blocks)."""
    g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
    p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
    cap = max(1, g.size)
    out = np.zeros(4 * cap, dtype=np.float64)
    nb = I64(0)
    check(lib().kt_plan_blocks(n_qubits, ptr(g), g.size, ptr(p), 0 if p is None else p.size, ptr(out), cap,
                               C.byref(nb)))
    return out[: 4 * nb.value].reshape(-1, 4)


def jit_stats() -> dict:
    """Run-time compiled block kernels so far, launches through them, and whether compiling failed."""
    k, l, f = I64(0), I64(0), I32(0)
    check(lib().kt_jit_stats(C.byref(k), C.byref(l), C.byref(f)))
    return {"kernels": int(k.value), "launches": int(l.value), "failed": bool(f.value)}


def jit_cache_stats() -> dict:
    """NVRTC compiles run in this process, and cubins loaded from KT_JIT_CACHE_DIR instead."""
    c, h = I64(0), I64(0)
    check(lib().kt_jit_cache_stats(C.byref(c), C.byref(h)))
    return {"nvrtc_compiles": int(c.value), "disk_hits": int(h.value)}


def jit_compile_only(n_qubits: int, gates: np.ndarray, params: np.ndarray | None = None, dtype: int = KT_C128) -> int:
    """Host-only: compile the run-time block kernels of an apply (no GPU); returns the block count."""
    g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
    p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
    k = I64(0)
    check(lib().kt_jit_compile_only(n_qubits, dtype, ptr(g), g.size, ptr(p), 0 if p is None else p.size, C.byref(k)))
    return int(k.value)


def tuning_set(name: str, value: int) -> None:
    check(lib().kt_tuning_set(name.encode(), int(value)))


def tuning_get(name: str) -> int:
    v = I64(0)
    check(lib().kt_tuning_get(name.encode(), C.byref(v)))
    return int(v.value)


def as_complex_interleaved(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a


class Statevector:
    """Device statevector handle (kt_sv)."""

    def __init__(self, n_qubits: int, dtype: int = KT_C128, stream: int | None = None):
        h = P()
        check(lib().kt_sv_create(n_qubits, dtype, C.byref(h)))
        self._h = h
        self.n_qubits = n_qubits
        self.dtype = dtype
        if stream is not None:
            check(lib().kt_sv_set_stream(self._h, stream))

    @classmethod
    def wrap(cls, device_ptr: int, n_qubits: int, dtype: int = KT_C128) -> "Statevector":
        self = cls.__new__(cls)
        h = P()
        check(lib().kt_sv_wrap(device_ptr, n_qubits, dtype, C.byref(h)))
        self._h = h
        self.n_qubits = n_qubits
        self.dtype = dtype
        return self

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            lib().kt_sv_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream: int | None):
        check(lib().kt_sv_set_stream(self._h, stream))

    def set_basis(self, index: int = 0):
        check(lib().kt_sv_set_basis(self._h, index))

    def upload(self, amps: np.ndarray):
        a = as_complex_interleaved(amps)
        check(lib().kt_sv_upload(self._h, ptr(a), a.size))

    def download(self) -> np.ndarray:
        out = np.empty(1 << self.n_qubits, dtype=np.complex128)
        check(lib().kt_sv_download(self._h, ptr(out), out.size))
        return out

    def copy_from(self, other: "Statevector"):
        check(lib().kt_sv_copy(self._h, other._h))

    def apply(self, gates: np.ndarray, params: np.ndarray | None = None, mode: int = KT_APPLY_FUSED):
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
        check(lib().kt_sv_apply(self._h, ptr(g), g.size, ptr(p), 0 if p is None else p.size, mode))

    def apply_stats(self):
        n = I64(0)
        b = C.c_double(0.0)
        check(lib().kt_sv_apply_stats(self._h, C.byref(n), C.byref(b)))
        return int(n.value), float(b.value)

    def expect(self, strings: np.ndarray, coeffs: np.ndarray | None = None):
        s = np.ascontiguousarray(strings, dtype=PAULI_DTYPE)
        c = None if coeffs is None else np.ascontiguousarray(coeffs, dtype=np.complex128)
        terms = np.empty(s.size, dtype=np.complex128)
        total = np.empty(1, dtype=np.complex128)
        check(lib().kt_sv_expect(self._h, ptr(s), s.size, ptr(c), ptr(terms), ptr(total)))
        return terms, complex(total[0])

    def probabilities(self, noise: np.ndarray | None = None) -> np.ndarray:
        out = np.empty(1 << self.n_qubits, dtype=np.float64)
        nz = None if noise is None else np.ascontiguousarray(noise, dtype=np.float64)
        check(lib().kt_sv_probabilities(self._h, ptr(nz), ptr(out)))
        return out

    def sample(self, canonicals: np.ndarray, noise: np.ndarray | None = None, mode: int = 0):
        c = np.ascontiguousarray(canonicals, dtype=np.float64)
        out = np.empty(c.size, dtype=np.uint64)
        nz = None if noise is None else np.ascontiguousarray(noise, dtype=np.float64)
        resc = I32(0)
        check(lib().kt_sv_sample(self._h, ptr(nz), ptr(c), c.size, ptr(out), mode, C.byref(resc)))
        return out, int(resc.value)

    def measure_probs(self, qubit: int):
        p0 = C.c_double()
        p1 = C.c_double()
        check(lib().kt_sv_measure_probs(self._h, qubit, C.byref(p0), C.byref(p1)))
        return p0.value, p1.value

    def collapse(self, qubit: int, outcome: int, scale: float):
        check(lib().kt_sv_collapse(self._h, qubit, outcome, scale))

    def norm_sq(self) -> float:
        v = C.c_double()
        check(lib().kt_sv_norm_sq(self._h, C.byref(v)))
        return v.value

    def prepare(self, gates: np.ndarray, params: np.ndarray | None = None):
        """Compile the fused block kernels of this circuit now (kt_sv_prepare)."""
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
        check(lib().kt_sv_prepare(self._h, ptr(g), g.size, ptr(p), 0 if p is None else p.size))

    def device_ptr(self) -> int:
        """Device address of the amplitudes (kt_sv_info)."""
        n, dt, p = I32(), I32(), P()
        check(lib().kt_sv_info(self._h, C.byref(n), C.byref(dt), C.byref(p)))
        return int(p.value)

    def inner(self, ket: "Statevector") -> complex:
        out = np.empty(2, dtype=np.float64)
        check(lib().kt_sv_inner(self._h, ket._h, ptr(out)))
        return complex(out[0], out[1])


    def tensor_product(self, right: "Statevector") -> "Statevector":
        """|self> (x) |right>, this state's qubits the low ones (kt_sv_tensor_product)."""
        out = Statevector(self.n_qubits + right.n_qubits, self.dtype)
        check(lib().kt_sv_tensor_product(self._h, right._h, out._h))
        return out

    def diagonal_expectation(self, eigenvalues) -> complex:
        """sum_i conj(psi_i) lambda_i psi_i (kt_sv_diagonal_expectation)."""
        lam = np.ascontiguousarray(eigenvalues, dtype=np.complex128)
        if lam.size != 1 << self.n_qubits:
            raise ValueError("one eigenvalue per basis state")
        out = np.empty(2, dtype=np.float64)
        check(lib().kt_sv_diagonal_expectation(self._h, ptr(lam), ptr(out)))
        return complex(out[0], out[1])

    def apply_dense5(self, u, passes: int = 3):
        """The 32 x 32 unitary `u` on qubits 0..4 of a complex64 state, on the tensor cores (kt_sv_apply_dense5;
        passes 3 or 4: TF32 split products of about FP32 accuracy, 1: plain TF32)."""
        m = np.ascontiguousarray(u, dtype=np.complex128)
        if m.shape != (32, 32):
            raise ValueError("u must be 32 x 32")
        check(lib().kt_sv_apply_dense5(self._h, ptr(m), passes))


def sample_probabilities(probabilities, canonicals, mode: int = 0, stream: int | None = None) -> np.ndarray:
    """Shots from a probability vector through the device sampler (kt_sample_probabilities)."""
    p = np.ascontiguousarray(probabilities, dtype=np.float64)
    c = np.ascontiguousarray(canonicals, dtype=np.float64)
    out = np.empty(c.size, dtype=np.uint64)
    check(lib().kt_sample_probabilities(ptr(p), p.size, ptr(c), c.size, ptr(out), mode, stream))
    return out


class DensityMatrix:
    """Device density-matrix handle (kt_dm): column-major N x N."""

    def __init__(self, n_qubits: int, dtype: int = KT_C128):
        h = P()
        check(lib().kt_dm_create(n_qubits, dtype, C.byref(h)))
        self._h = h
        self.n_qubits = n_qubits
        self.dtype = dtype

    def close(self):
        if getattr(self, "_h", None):
            lib().kt_dm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream: int | None):
        check(lib().kt_dm_set_stream(self._h, stream))

    def set_basis(self, index: int = 0):
        check(lib().kt_dm_set_basis(self._h, index))

    def upload(self, rho: np.ndarray):
        """rho: (N, N) complex matrix (any memory order); stored column-major."""
        a = np.ascontiguousarray(np.asarray(rho, dtype=np.complex128).T).reshape(-1)
        check(lib().kt_dm_upload(self._h, ptr(a), a.size))

    def download(self) -> np.ndarray:
        N = 1 << self.n_qubits
        flat = np.empty(N * N, dtype=np.complex128)
        check(lib().kt_dm_download(self._h, ptr(flat), flat.size))
        return flat.reshape(N, N).T.copy()  # column-major -> (row, col)

    def apply(self, gates: np.ndarray, params: np.ndarray | None = None, mode: int = KT_APPLY_FUSED):
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
        check(lib().kt_dm_apply(self._h, ptr(g), g.size, ptr(p), 0 if p is None else p.size, mode))

    def prepare(self, gates: np.ndarray, params: np.ndarray | None = None):
        """Compile the fused block kernels of this circuit on the density matrix now (kt_dm_prepare)."""
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
        check(lib().kt_dm_prepare(self._h, ptr(g), g.size, ptr(p), 0 if p is None else p.size))

    def measure_probs(self, qubit: int):
        """P(0), P(1) of an M gate on `qubit` as the reference defines them (kt_dm_measure_probs)."""
        p0 = C.c_double()
        p1 = C.c_double()
        check(lib().kt_dm_measure_probs(self._h, qubit, C.byref(p0), C.byref(p1)))
        return p0.value, p1.value

    def collapse(self, qubit: int, outcome: int, scale: float):
        check(lib().kt_dm_collapse(self._h, qubit, outcome, scale))

    def apply_stats(self):
        n = I64(0)
        b = C.c_double(0.0)
        check(lib().kt_dm_apply_stats(self._h, C.byref(n), C.byref(b)))
        return int(n.value), float(b.value)

    def expect(self, strings: np.ndarray, coeffs: np.ndarray | None = None):
        s = np.ascontiguousarray(strings, dtype=PAULI_DTYPE)
        c = None if coeffs is None else np.ascontiguousarray(coeffs, dtype=np.complex128)
        terms = np.empty(s.size, dtype=np.complex128)
        total = np.empty(1, dtype=np.complex128)
        check(lib().kt_dm_expect(self._h, ptr(s), s.size, ptr(c), ptr(terms), ptr(total)))
        return terms, complex(total[0])

    def trace(self) -> complex:
        out = np.empty(2, dtype=np.float64)
        check(lib().kt_dm_trace(self._h, ptr(out)))
        return complex(out[0], out[1])

    def probabilities(self) -> np.ndarray:
        out = np.empty(1 << self.n_qubits, dtype=np.float64)
        check(lib().kt_dm_probabilities(self._h, ptr(out)))
        return out

    def partial_trace(self, qubits) -> "DensityMatrix":
        """A new density matrix: this one traced over `qubits` (distinct), in
        the order given (sums grouped like tracing one qubit at a time)."""
        q = np.ascontiguousarray(list(qubits), dtype=np.int32)
        out = DensityMatrix(self.n_qubits - q.size, self.dtype)
        check(lib().kt_dm_partial_trace(self._h, ptr(q), q.size, out._h))
        return out

    def tensor_product(self, right: "DensityMatrix") -> "DensityMatrix":
        """self (low qubits) (x) right (high qubits)."""
        out = DensityMatrix(self.n_qubits + right.n_qubits, self.dtype)
        check(lib().kt_dm_tensor_product(self._h, right._h, out._h))
        return out

    def trace_of_square(self) -> complex:
        out = np.empty(2, dtype=np.float64)
        check(lib().kt_dm_trace_of_square(self._h, ptr(out)))
        return complex(out[0], out[1])


def pairs_single(n: int, t: int, k0: int = 0, count: int | None = None) -> np.ndarray:
    if count is None:
        count = (1 << (n - 1)) - k0
    out = np.empty((count, 2), dtype=np.uint64)
    check(lib().kt_pairs_single(n, t, k0, count, ptr(out)))
    return out


def pairs_double(n: int, c: int, t: int, quad: bool = False, k0: int = 0, count: int | None = None) -> np.ndarray:
    if count is None:
        count = (1 << (n - 2)) - k0
    out = np.empty((count, 4 if quad else 2), dtype=np.uint64)
    check(lib().kt_pairs_double(n, c, t, 1 if quad else 0, k0, count, ptr(out)))
    return out


class Adjoint:
    """Adjoint gradient of E = Re <psi|H|psi> for a parameterised circuit (kt_adjoint).

    forward() runs the circuit on the given statevector (from its current
    state) and returns E; backward() returns dE/dparams and leaves the
    statevector un-applied back to its initial state."""

    def __init__(self, sv: Statevector, checkpoint_every: int = 0):
        h = P()
        check(lib().kt_adjoint_create(sv.handle, checkpoint_every, C.byref(h)))
        self._h = h
        self.sv = sv
        self.n_params = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().kt_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, gates, params, strings, coeffs=None) -> float:
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        p = np.ascontiguousarray(params, dtype=np.float64)
        s = np.ascontiguousarray(strings, dtype=PAULI_DTYPE)
        c = None if coeffs is None else np.ascontiguousarray(coeffs, dtype=np.complex128)
        e = C.c_double()
        check(lib().kt_adjoint_forward(self._h, ptr(g), g.size, ptr(p), p.size, ptr(s), s.size, ptr(c), C.byref(e)))
        self.n_params = p.size
        return e.value

    def backward(self) -> np.ndarray:
        out = np.zeros(self.n_params, dtype=np.float64)
        check(lib().kt_adjoint_backward(self._h, ptr(out), out.size))
        return out


def batch_items(circuits) -> tuple:
    """Concatenate per-item (n_qubits, gates, n_params, strings, coeffs) into the
    flat arrays kt_batch_create takes: (items, gates, strings, coeffs, n_params_total).
    Each item's parameters follow the previous item's (disjoint ranges)."""
    items = np.zeros(len(circuits), dtype=BATCH_ITEM_DTYPE)
    g_parts, s_parts, c_parts = [], [], []
    g_off = p_off = s_off = 0
    for b, (n, gates, n_params, strings, coeffs) in enumerate(circuits):
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        s = np.ascontiguousarray(strings, dtype=PAULI_DTYPE)
        c = np.ones(s.size, dtype=np.complex128) if coeffs is None else np.asarray(coeffs, dtype=np.complex128)
        items[b] = (n, 0, g_off, g.size, p_off, n_params, s_off, s.size)
        g_parts.append(g)
        s_parts.append(s)
        c_parts.append(c)
        g_off += g.size
        p_off += n_params
        s_off += s.size
    gates = np.concatenate(g_parts) if g_parts else np.zeros(0, dtype=GATE_DTYPE)
    return items, gates, np.concatenate(s_parts), np.concatenate(c_parts), p_off


class Batch:
    """Energies (and adjoint gradients) of many independent circuits (kt_batch).

    `items` is a BATCH_ITEM_DTYPE array over the flat `gates`, `strings` and
    `coeffs` arrays (see batch_items); planning, allocation and the CUDA graph
    happen here, evaluate() replays the graph for a parameter vector."""

    def __init__(self, items, gates, strings, coeffs, n_params: int, dtype: int = KT_C128, with_grad: bool = True):
        it = np.ascontiguousarray(items, dtype=BATCH_ITEM_DTYPE)
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        s = np.ascontiguousarray(strings, dtype=PAULI_DTYPE)
        c = None if coeffs is None else np.ascontiguousarray(coeffs, dtype=np.complex128)
        h = P()
        check(lib().kt_batch_create(ptr(it), it.size, ptr(g), g.size, int(n_params), ptr(s), ptr(c), s.size, dtype,
                                    1 if with_grad else 0, C.byref(h)))
        self._h = h
        self.n_items = it.size
        self.n_params = int(n_params)
        self.with_grad = with_grad

    def close(self):
        if getattr(self, "_h", None):
            lib().kt_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream: int | None):
        check(lib().kt_batch_set_stream(self._h, stream))

    def evaluate(self, params) -> tuple:
        p = np.ascontiguousarray(params, dtype=np.float64)
        if p.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {p.size}")
        e = np.empty(self.n_items, dtype=np.float64)
        g = np.empty(self.n_params, dtype=np.float64) if self.with_grad else None
        check(lib().kt_batch_evaluate(self._h, ptr(p), ptr(e), ptr(g)))
        return e, g

    def stats(self) -> dict:
        v = [I64() for _ in range(6)]
        a, d = C.c_double(), C.c_double()
        check(lib().kt_batch_stats(self._h, *[C.byref(x) for x in v], C.byref(a), C.byref(d)))
        keys = ("small_items", "large_items", "waves", "jobs", "units", "launches")
        out = {k: x.value for k, x in zip(keys, v)}
        out["alg_bytes"] = a.value
        out["device_bytes"] = d.value
        cl, ci = I64(), I64()
        check(lib().kt_batch_compiled(self._h, C.byref(cl), C.byref(ci)))
        out["compiled_classes"] = cl.value
        out["compiled_items"] = ci.value
        return out
