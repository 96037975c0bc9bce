"""Python loader for the oracle — TEST INFRASTRUCTURE ONLY.

Two checkers, both CPU:
  * `port`: oracle/libkt_oracle.so, the C restatement of the reference
    algorithms (oracle/kt_oracle.c);
  * `ref`:  oracle/_ref/libkettle_ref.so, the reference library itself built
    from its sources (oracle/Makefile), through oracle/ref_capi.cpp.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  The product never does.
"""
from __future__ import annotations

import ctypes as C
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
PORT_PATH = HERE / "libkt_oracle.so"
REF_PATH = HERE / "_ref" / "libkettle_ref.so"

P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64
U32 = C.c_uint32
U64 = C.c_uint64

GATE_DTYPE = np.dtype([("op", "u1"), ("r0", "u1"), ("r1", "<u2"), ("target", "<u4"), ("control", "<u4"),
                       ("param", "<i4"), ("angle", "<f8"), ("u", "<f8", (8,))], align=True)
PAULI_DTYPE = np.dtype([("x", "<u8"), ("z", "<u8"), ("phase", "<i4"), ("r", "<i4")], align=True)


def _p(a):
    return None if a is None else a.ctypes.data


def _build_port():
    subprocess.run(["make", "-s", "-C", str(HERE), "port"], check=True, capture_output=True)


class Port:
    """The C restatement (always available: it is built from oracle/kt_oracle.c)."""

    def __init__(self):
        if not PORT_PATH.exists() or PORT_PATH.stat().st_mtime < (HERE / "kt_oracle.c").stat().st_mtime:
            _build_port()
        L = C.CDLL(str(PORT_PATH))
        L.kto_pairs_single.argtypes = [U32, U32, U64, U64, P]
        L.kto_pairs_double.argtypes = [U32, U32, U32, I32, U64, U64, P]
        L.kto_apply.argtypes = [I32, P, P, I64, P]
        L.kto_apply.restype = I32
        L.kto_expect.argtypes = [I32, P, P, I64, P, P, P]
        L.kto_expect.restype = I32
        L.kto_probabilities.argtypes = [I32, P, P, P]
        L.kto_probabilities.restype = I32
        L.kto_canonicals_mt19937.argtypes = [U32, I64, P]
        L.kto_canonicals_mt19937.restype = I32
        L.kto_sample.argtypes = [I32, P, P, I64, P]
        L.kto_sample.restype = I32
        L.kto_sample_raw.argtypes = [P, U64, P, I64, P]
        L.kto_sample_raw.restype = I32
        L.kto_measure.argtypes = [I32, P, U32, C.c_double, C.POINTER(I32), C.POINTER(C.c_double),
                                  C.POINTER(C.c_double)]
        L.kto_measure.restype = I32
        L.kto_simulate_dm.argtypes = [I32, P, P, I64, P]
        L.kto_simulate_dm.restype = I32
        L.kto_dm_expect.argtypes = [I32, P, P, I64, P, P, P]
        L.kto_dm_expect.restype = I32
        L.kto_gate_matrix.argtypes = [P, P, P]
        L.kto_dm_partial_trace.argtypes = [I32, P, P, I32, P]
        L.kto_dm_partial_trace.restype = I32
        L.kto_dm_tensor_product.argtypes = [I32, P, I32, P, P]
        L.kto_dm_tensor_product.restype = I32
        L.kto_dm_trace_of_square.argtypes = [I32, P, P]
        L.kto_dm_trace_of_square.restype = I32
        self.L = L

    def pairs_single(self, n, t, k0=0, count=None):
        count = (1 << (n - 1)) - k0 if count is None else count
        out = np.empty((count, 2), dtype=np.uint64)
        self.L.kto_pairs_single(n, t, k0, count, _p(out))
        return out

    def pairs_double(self, n, c, t, quad=False, k0=0, count=None):
        count = (1 << (n - 2)) - k0 if count is None else count
        out = np.empty((count, 4 if quad else 2), dtype=np.uint64)
        self.L.kto_pairs_double(n, c, t, 1 if quad else 0, k0, count, _p(out))
        return out

    def apply(self, n, amps, gates, params=None):
        a = np.array(amps, dtype=np.complex128, copy=True)
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
        rc = self.L.kto_apply(n, _p(a), _p(g), g.size, _p(p))
        if rc != 0:
            raise ValueError("oracle rejected the gate stream")
        return a

    def expect(self, n, amps, strings, coeffs=None):
        a = np.ascontiguousarray(amps, dtype=np.complex128)
        s = np.ascontiguousarray(strings, dtype=PAULI_DTYPE)
        c = None if coeffs is None else np.ascontiguousarray(coeffs, dtype=np.complex128)
        terms = np.empty(s.size, dtype=np.complex128)
        total = np.empty(1, dtype=np.complex128)
        self.L.kto_expect(n, _p(a), _p(s), s.size, _p(c), _p(terms), _p(total))
        return terms, complex(total[0])

    def probabilities(self, n, amps, noise=None):
        a = np.ascontiguousarray(amps, dtype=np.complex128)
        out = np.empty(1 << n, dtype=np.float64)
        nz = None if noise is None else np.ascontiguousarray(noise, dtype=np.float64)
        self.L.kto_probabilities(n, _p(a), _p(nz), _p(out))
        return out

    def canonicals(self, seed, count):
        out = np.empty(count, dtype=np.float64)
        self.L.kto_canonicals_mt19937(seed & 0xFFFFFFFF, count, _p(out))
        return out

    def sample(self, n, probs, canonicals):
        pr = np.ascontiguousarray(probs, dtype=np.float64)
        c = np.ascontiguousarray(canonicals, dtype=np.float64)
        out = np.empty(c.size, dtype=np.uint64)
        rc = self.L.kto_sample(n, _p(pr), _p(c), c.size, _p(out))
        if rc != 0:
            raise ValueError("oracle sampling failed")
        return out

    def sample_raw(self, probs, canonicals):
        """Sampling from any probability vector (the std::vector<double> overloads)."""
        pr = np.ascontiguousarray(probs, dtype=np.float64)
        c = np.ascontiguousarray(canonicals, dtype=np.float64)
        out = np.empty(c.size, dtype=np.uint64)
        if self.L.kto_sample_raw(_p(pr), pr.size, _p(c), c.size, _p(out)) != 0:
            raise ValueError("oracle sampling failed")
        return out

    def measure(self, n, amps, qubit, canonical):
        a = np.array(amps, dtype=np.complex128, copy=True)
        o = I32()
        p0 = C.c_double()
        p1 = C.c_double()
        self.L.kto_measure(n, _p(a), qubit, canonical, C.byref(o), C.byref(p0), C.byref(p1))
        return a, int(o.value), p0.value, p1.value

    def simulate_dm(self, n, rho, gates, params=None):
        """rho: (N, N) complex -> evolved (N, N)."""
        flat = np.ascontiguousarray(np.asarray(rho, dtype=np.complex128).T).reshape(-1).copy()
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
        rc = self.L.kto_simulate_dm(n, _p(flat), _p(g), g.size, _p(p))
        if rc != 0:
            raise ValueError("oracle rejected the gate stream")
        N = 1 << n
        return flat.reshape(N, N).T.copy()

    def dm_expect(self, n, rho, strings, coeffs=None):
        flat = np.ascontiguousarray(np.asarray(rho, dtype=np.complex128).T).reshape(-1)
        s = np.ascontiguousarray(strings, dtype=PAULI_DTYPE)
        c = None if coeffs is None else np.ascontiguousarray(coeffs, dtype=np.complex128)
        terms = np.empty(s.size, dtype=np.complex128)
        total = np.empty(1, dtype=np.complex128)
        self.L.kto_dm_expect(n, _p(flat), _p(s), s.size, _p(c), _p(terms), _p(total))
        return terms, complex(total[0])

    def dm_partial_trace(self, n, rho, qubits):
        """rho (N, N) -> the reduced (M, M), qubits read as the reference reads them."""
        flat = np.ascontiguousarray(np.asarray(rho, dtype=np.complex128).T).reshape(-1)
        q = np.ascontiguousarray(list(qubits), dtype=np.int64)
        m = n - q.size
        out = np.empty((1 << m) * (1 << m), dtype=np.complex128)
        self._chk_dm(self.L.kto_dm_partial_trace(n, _p(flat), _p(q), q.size, _p(out)))
        return out.reshape(1 << m, 1 << m).T.copy()

    def dm_tensor_product(self, nl, left, nr, right):
        l = np.ascontiguousarray(np.asarray(left, dtype=np.complex128).T).reshape(-1)
        r = np.ascontiguousarray(np.asarray(right, dtype=np.complex128).T).reshape(-1)
        D = 1 << (nl + nr)
        out = np.empty(D * D, dtype=np.complex128)
        self._chk_dm(self.L.kto_dm_tensor_product(nl, _p(l), nr, _p(r), _p(out)))
        return out.reshape(D, D).T.copy()

    def dm_trace_of_square(self, n, rho):
        flat = np.ascontiguousarray(np.asarray(rho, dtype=np.complex128).T).reshape(-1)
        out = np.empty(2, dtype=np.float64)
        self._chk_dm(self.L.kto_dm_trace_of_square(n, _p(flat), _p(out)))
        return complex(out[0], out[1])

    @staticmethod
    def _chk_dm(rc):
        if rc != 0:
            raise ValueError("oracle rejected the density-matrix operation")

    def gate_matrix(self, gate_rec, params=None):
        g = np.ascontiguousarray(gate_rec, dtype=GATE_DTYPE).reshape(1)
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
        m = np.empty(8, dtype=np.float64)
        self.L.kto_gate_matrix(_p(g), _p(p), _p(m))
        return np.array([[m[0] + 1j * m[1], m[2] + 1j * m[3]], [m[4] + 1j * m[5], m[6] + 1j * m[7]]])


class Ref:
    """The reference library compiled from its own sources (oracle/_ref)."""

    def __init__(self):
        if not REF_PATH.exists():
            raise FileNotFoundError(f"{REF_PATH} not built (make -C oracle ref)")
        L = C.CDLL(str(REF_PATH))
        L.ref_last_error.restype = C.c_char_p
        L.ref_simulate_sv.argtypes = [I32, P, I64, P, P, I64, P]
        L.ref_simulate_sv.restype = I32
        L.ref_simulate_dm.argtypes = [I32, P, I64, P, P, I64]
        L.ref_simulate_dm.restype = I32
        L.ref_sv_to_dm.argtypes = [I32, P, P]
        L.ref_sv_to_dm.restype = I32
        L.ref_expect_sv.argtypes = [I32, P, P, I64, P, P, P]
        L.ref_expect_sv.restype = I32
        L.ref_probabilities.argtypes = [I32, P, P, P]
        L.ref_probabilities.restype = I32
        L.ref_sample_memory.argtypes = [I32, P, P, I64, I64, P]
        L.ref_sample_memory.restype = I32
        L.ref_sample_counts.argtypes = [I32, P, I64, I64, P, I64]
        L.ref_sample_counts.restype = I32
        L.ref_pairs_single.argtypes = [U32, U32, U64, U64, P]
        L.ref_pairs_single.restype = I32
        L.ref_pairs_double.argtypes = [U32, U32, U32, I32, U64, U64, P]
        L.ref_pairs_double.restype = I32
        L.ref_random_unitary.argtypes = [I32, P]
        L.ref_random_unitary.restype = I32
        L.ref_random_unitaries.argtypes = [I32, I64, P]
        L.ref_random_unitaries.restype = I32
        L.ref_sample_probabilities.argtypes = [P, I64, I64, I64, P]
        L.ref_sample_probabilities.restype = I32
        L.ref_time_sv.argtypes = [I32, P, I64, P, C.POINTER(C.c_double)]
        L.ref_time_sv.restype = I32
        L.ref_sv_alloc.argtypes = [I32]
        L.ref_sv_alloc.restype = P
        L.ref_sv_free.argtypes = [P]
        L.ref_sv_time.argtypes = [P, P, I64, P, C.POINTER(C.c_double)]
        L.ref_sv_time.restype = I32
        L.ref_dm_partial_trace.argtypes = [I32, P, P, I32, P]
        L.ref_dm_partial_trace.restype = I32
        L.ref_dm_tensor_product.argtypes = [I32, P, I32, P, P]
        L.ref_dm_tensor_product.restype = I32
        L.ref_dm_trace_of_square.argtypes = [I32, P, P]
        L.ref_dm_trace_of_square.restype = I32
        self.L = L

    def time_sv(self, n, gates, params=None):
        """Seconds of ket::simulate on a fresh |0...0> of n qubits (state built outside the timing)."""
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
        s = C.c_double()
        self._chk(self.L.ref_time_sv(n, _p(g), g.size, _p(p), C.byref(s)))
        return s.value

    class Held:
        """A reference Statevector kept alive across timed ket::simulate calls."""

        def __init__(self, L, n):
            self.L = L
            self.h = L.ref_sv_alloc(n)
            if not self.h:
                raise MemoryError(L.ref_last_error().decode())

        def time(self, gates, params=None):
            g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
            p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
            s = C.c_double()
            if self.L.ref_sv_time(self.h, _p(g), g.size, _p(p), C.byref(s)) != 0:
                raise ValueError(self.L.ref_last_error().decode())
            return s.value

        def close(self):
            if self.h:
                self.L.ref_sv_free(self.h)
                self.h = None

    def held_state(self, n):
        return Ref.Held(self.L, n)

    def _chk(self, rc):
        if rc != 0:
            raise ValueError(self.L.ref_last_error().decode())

    def simulate_sv(self, n, amps, gates, params=None, seed=-1, n_bits=None):
        a = np.array(amps, dtype=np.complex128, copy=True)
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
        cb = np.full(n if n_bits is None else n_bits, -2, dtype=np.int32)
        self._chk(self.L.ref_simulate_sv(n, _p(g), g.size, _p(p), _p(a), seed, _p(cb)))
        return a, cb

    def simulate_dm(self, n, rho, gates, params=None, seed=-1):
        flat = np.ascontiguousarray(np.asarray(rho, dtype=np.complex128).T).reshape(-1).copy()
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
        self._chk(self.L.ref_simulate_dm(n, _p(g), g.size, _p(p), _p(flat), seed))
        N = 1 << n
        return flat.reshape(N, N).T.copy()

    def dm_partial_trace(self, n, rho, qubits):
        """rho (N, N) -> the reduced (M, M), qubits read as the reference reads them."""
        flat = np.ascontiguousarray(np.asarray(rho, dtype=np.complex128).T).reshape(-1)
        q = np.ascontiguousarray(list(qubits), dtype=np.int64)
        m = n - q.size
        out = np.empty((1 << m) * (1 << m), dtype=np.complex128)
        self._chk_dm(self.L.ref_dm_partial_trace(n, _p(flat), _p(q), q.size, _p(out)))
        return out.reshape(1 << m, 1 << m).T.copy()

    def dm_tensor_product(self, nl, left, nr, right):
        l = np.ascontiguousarray(np.asarray(left, dtype=np.complex128).T).reshape(-1)
        r = np.ascontiguousarray(np.asarray(right, dtype=np.complex128).T).reshape(-1)
        D = 1 << (nl + nr)
        out = np.empty(D * D, dtype=np.complex128)
        self._chk_dm(self.L.ref_dm_tensor_product(nl, _p(l), nr, _p(r), _p(out)))
        return out.reshape(D, D).T.copy()

    def dm_trace_of_square(self, n, rho):
        flat = np.ascontiguousarray(np.asarray(rho, dtype=np.complex128).T).reshape(-1)
        out = np.empty(2, dtype=np.float64)
        self._chk_dm(self.L.ref_dm_trace_of_square(n, _p(flat), _p(out)))
        return complex(out[0], out[1])

    def _chk_dm(self, rc):
        self._chk(rc)

    def sv_to_dm(self, n, amps):
        a = np.ascontiguousarray(amps, dtype=np.complex128)
        N = 1 << n
        flat = np.empty(N * N, dtype=np.complex128)
        self._chk(self.L.ref_sv_to_dm(n, _p(a), _p(flat)))
        return flat.reshape(N, N).T.copy()

    def expect(self, n, amps, strings, coeffs=None):
        a = np.ascontiguousarray(amps, dtype=np.complex128)
        s = np.ascontiguousarray(strings, dtype=PAULI_DTYPE)
        c = None if coeffs is None else np.ascontiguousarray(coeffs, dtype=np.complex128)
        terms = np.empty(s.size, dtype=np.complex128)
        total = np.empty(1, dtype=np.complex128)
        self._chk(self.L.ref_expect_sv(n, _p(a), _p(s), s.size, _p(c), _p(terms), _p(total)))
        return terms, complex(total[0])

    def probabilities(self, n, amps, noise=None):
        a = np.ascontiguousarray(amps, dtype=np.complex128)
        out = np.empty(1 << n, dtype=np.float64)
        nz = None if noise is None else np.ascontiguousarray(noise, dtype=np.float64)
        self._chk(self.L.ref_probabilities(n, _p(a), _p(nz), _p(out)))
        return out

    def sample_memory(self, n, amps, n_shots, seed, noise=None):
        a = np.ascontiguousarray(amps, dtype=np.complex128)
        out = np.empty(n_shots, dtype=np.uint64)
        nz = None if noise is None else np.ascontiguousarray(noise, dtype=np.float64)
        self._chk(self.L.ref_sample_memory(n, _p(a), _p(nz), n_shots, seed, _p(out)))
        return out

    def sample_counts(self, n, amps, n_shots, seed):
        a = np.ascontiguousarray(amps, dtype=np.complex128)
        buf = C.create_string_buffer(64 * (n + 16) * min(n_shots, 1 << n) + 64)
        self._chk(self.L.ref_sample_counts(n, _p(a), n_shots, seed, buf, len(buf)))
        out = {}
        for line in buf.value.decode().splitlines():
            k, v = line.split()
            out[k] = int(v)
        return out

    def pairs_single(self, n, t, k0=0, count=None):
        count = (1 << (n - 1)) - k0 if count is None else count
        out = np.empty((count, 2), dtype=np.uint64)
        self._chk(self.L.ref_pairs_single(n, t, k0, count, _p(out)))
        return out

    def pairs_double(self, n, c, t, quad=False, k0=0, count=None):
        count = (1 << (n - 2)) - k0 if count is None else count
        out = np.empty((count, 4 if quad else 2), dtype=np.uint64)
        self._chk(self.L.ref_pairs_double(n, c, t, 1 if quad else 0, k0, count, _p(out)))
        return out

    def random_unitary(self, seed):
        u = np.empty(8, dtype=np.float64)
        self._chk(self.L.ref_random_unitary(seed, _p(u)))
        return np.array([[u[0] + 1j * u[1], u[2] + 1j * u[3]], [u[4] + 1j * u[5], u[6] + 1j * u[7]]])

    def sample_probabilities(self, probs, n_shots, seed):
        p = np.ascontiguousarray(probs, dtype=np.float64)
        out = np.empty(n_shots, dtype=np.uint64)
        self._chk(self.L.ref_sample_probabilities(_p(p), p.size, n_shots, seed, _p(out)))
        return out

    def random_unitaries(self, seed, count):
        """`count` matrices of generate_random_unitary2x2 on one std::mt19937(seed) stream."""
        u = np.empty(8 * count, dtype=np.float64)
        self._chk(self.L.ref_random_unitaries(seed, count, _p(u)))
        return [np.array([[u[8 * k] + 1j * u[8 * k + 1], u[8 * k + 2] + 1j * u[8 * k + 3]],
                          [u[8 * k + 4] + 1j * u[8 * k + 5], u[8 * k + 6] + 1j * u[8 * k + 7]]]) for k in range(count)]


_port = None
_ref = None


def port() -> Port:
    global _port
    if _port is None:
        _port = Port()
    return _port


def ref() -> Ref:
    global _ref
    if _ref is None:
        _ref = Ref()
    return _ref


def ref_available() -> bool:
    return REF_PATH.exists()
