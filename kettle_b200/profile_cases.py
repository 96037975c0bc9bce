"""Small, self-contained workloads that run one family of the engine's kernels
a few times, for profiling them one at a time (for example under Nsight
Compute with a kernel-name filter and a launch count):

    python -m kettle_b200.profile_cases <case> [--qubits N] [--reps R]

Every case first runs its operation once (warm-up: plans, compiled kernels,
scratch buffers), then `reps` more times, so a profiler can skip the first
launch of the kernel it captures.  The states are sized past the 126 MB L2
(1 GiB by default) so DRAM figures mean something, and stay a few GB at most.

Cases and the kernels they run:
  pauli        k_pauli, k_pauli_finalize          (kt_sv_expect, 32 strings)
  sample       k_probs_tiles, k_tile_*, k_exact_chain, k_bound_tile, k_sparse_bound, k_shot_*
               (kt_sv_sample, exact tier, on a dense state)
  sample_fast  k_probs, k_chunk_sums, k_chunk_offsets, k_sample_bound, k_sample_fast  (2^22 amplitudes)
  dm_pauli     k_dm_pauli, k_dm_pauli_finalize    (kt_dm_expect on a 13-qubit density matrix)
  hpsi         k_hsum                              (lambda = H psi and the energy, in the adjoint forward)
  adjoint      k_fused_adj, k_adj_rows             (fused adjoint backward blocks)
  dm_ops       k_partial_trace, k_tensor_product, k_trace_square
  norm         compiled blocks (prepared plan; k_fused_norm with fused_jit=0), k_norm_final
               (complex64 renormalising apply)
  blocks       kt_jb* (run-time compiled blocks of the benchmark circuit family)
  fused        k_fused (the precompiled fused-block interpreter)
  sweep        k_sweep (one pass per gate)
  state_ops    k_sv_tensor_product, k_sv_diag_expect, k_dm_block_norms, k_dm_collapse
  batch        k_batch_persist, k_batch_small, k_batch_patch (batch_jit_min_qubits=0: the interpreted blocks)
  batch_class  kt_jbb*, kt_jab*, k_batch_ham_items, k_batch_basis: one compiled class of 48 items
               (20 qubits, 4 layers, 20 strings: 768 MiB of states per launch)
  dense_block  the tensor-core question: 40 random gates on qubits 0..4 of a
               complex64 state applied by the engine (one fused pass of
               compiled SIMT blocks) against the same 32 x 32 unitary applied
               as a dense GEMM: by the engine's own tcgen05 kernel
               (kt_sv_apply_dense5: four, three and one TF32 products) and by
               cuBLAS through torch, in FP32 on the CUDA cores and in TF32
               on the tensor cores; prints times (CUDA
               events, best of reps) and the largest amplitude error of each
               against the complex128 engine result
"""
from __future__ import annotations

import argparse
import sys

import numpy as np

from . import capi
from . import workloads as W


def _random_state(n, seed, dtype=capi.KT_C128):
    sv = capi.Statevector(n, dtype)
    sv.set_basis(0)
    sv.apply(W.random_layers(n, 1, seed=seed, mixed=True))
    return sv


def case_pauli(n, reps):
    sv = _random_state(n, 1)
    strings, coeffs = W.random_paulis(n, 32, seed=2)
    for _ in range(1 + reps):
        sv.expect(strings, coeffs)
    sv.close()


def case_sample(n, reps):
    # eight mixed layers: a dense, Porter-Thomas-like distribution, as the
    # benchmark circuit's final state is
    sv = capi.Statevector(n)
    sv.set_basis(0)
    sv.apply(W.random_layers(n, 8, seed=3, mixed=True))
    can = capi.canonicals_mt19937(4, 4096)
    for _ in range(1 + reps):
        sv.sample(can)
    sv.close()


def case_sample_fast(n, reps):
    case_sample(min(n, 22), reps)


def case_dm_pauli(n, reps):
    m = max(2, n // 2)
    dm = capi.DensityMatrix(m)
    dm.apply(W.random_layers(m, 2, seed=5, mixed=True))
    strings, coeffs = W.random_paulis(m, 32, seed=6)
    for _ in range(1 + reps):
        dm.expect(strings, coeffs)
    dm.close()


def case_hpsi(n, reps):
    gates, params = W.hea(n, 1, seed=7)
    strings, coeffs = W.xxz_chain(n, seed=7)
    sv = capi.Statevector(n)
    adj = capi.Adjoint(sv)
    for _ in range(1 + reps):
        sv.set_basis(0)
        adj.forward(gates, params, strings, coeffs)
        adj.backward()
    adj.close()
    sv.close()


def case_adjoint(n, reps):
    gates, params = W.hea(n, 2, seed=8)
    strings, coeffs = W.xxz_chain(n, seed=8)
    sv = capi.Statevector(n)
    adj = capi.Adjoint(sv)
    for _ in range(1 + reps):
        sv.set_basis(0)
        adj.forward(gates, params, strings, coeffs)
        adj.backward()
    adj.close()
    sv.close()


def case_dm_ops(n, reps):
    m = max(2, n // 2)
    dm = capi.DensityMatrix(m)
    dm.apply(W.random_layers(m, 2, seed=9, mixed=True))
    left = capi.DensityMatrix(m // 2)
    right = capi.DensityMatrix(m - m // 2)
    for _ in range(1 + reps):
        dm.partial_trace([0]).close()
        left.tensor_product(right).close()
        dm.trace_of_square()
    for h in (dm, left, right):
        h.close()


def case_norm(n, reps):
    g = W.random_layers(n, 2, seed=10, mixed=True)
    sv = capi.Statevector(n, capi.KT_C64)
    sv.prepare(g)
    for _ in range(1 + reps):
        sv.set_basis(0)
        sv.apply(g)
    sv.close()


def case_blocks(n, reps):
    g = W.random_layers(n, 2, seed=2024, mixed=True)
    sv = capi.Statevector(n)
    sv.prepare(g)
    for _ in range(1 + reps):
        sv.set_basis(0)
        sv.apply(g)
    sv.close()


def case_fused(n, reps):
    old = capi.tuning_get("fused_jit")
    capi.tuning_set("fused_jit", 0)
    try:
        case_blocks(n, reps)
    finally:
        capi.tuning_set("fused_jit", old)


def case_sweep(n, reps):
    g = W.random_layers(n, 1, seed=11, mixed=True)[: 2 * n]
    sv = capi.Statevector(n)
    for _ in range(1 + reps):
        sv.set_basis(0)
        sv.apply(g, mode=capi.KT_APPLY_PER_GATE)
    sv.close()


def case_state_ops(n, reps):
    a = _random_state(n // 2, 12)
    b = _random_state(n - n // 2, 13)
    lam = np.linspace(-1.0, 1.0, 1 << n).astype(np.complex128)
    m = max(2, n // 2)
    dm = capi.DensityMatrix(m)
    dm.apply(W.random_layers(m, 1, seed=14, mixed=True))
    for _ in range(1 + reps):
        out = a.tensor_product(b)
        out.diagonal_expectation(lam)
        out.close()
        dm.measure_probs(1)
    dm.collapse(1, 0, 1.0)
    for h in (a, b, dm):
        h.close()


def case_batch(n, reps):
    circuits, params = W.hea_batch(64, seed=15, qubits=(10, min(n, 20)), layers=(2, 6), n_strings=20)
    items, gates, strings, coeffs, n_params = capi.batch_items(circuits)
    old = capi.tuning_get("batch_jit_min_qubits")
    capi.tuning_set("batch_jit_min_qubits", 0)
    try:
        b = capi.Batch(items, gates, strings, coeffs, n_params)
    finally:
        capi.tuning_set("batch_jit_min_qubits", old)
    for _ in range(1 + reps):
        b.evaluate(params)
    b.close()


def case_batch_class(n, reps):
    circuits, params = W.hea_batch(48, seed=16, qubits=(20, 20), layers=(4, 4), n_strings=20)
    items, gates, strings, coeffs, n_params = capi.batch_items(circuits)
    b = capi.Batch(items, gates, strings, coeffs, n_params)
    assert b.stats()["compiled_classes"] == 1
    for _ in range(1 + reps):
        b.evaluate(params)
    b.close()


class _DeviceArray:
    """A raw device buffer seen by torch (__cuda_array_interface__)."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3}


def case_dense_block(n, reps):
    import json

    import torch

    k = 5
    rng = np.random.default_rng(16)
    names = ["H", "RX", "RY", "RZ", "U", "CX", "CRY", "CP"]
    recs = []
    for _ in range(40):
        name = names[int(rng.integers(len(names)))]
        t = int(rng.integers(k))
        if name in ("CX", "CRY", "CP"):
            c = int((t + 1 + rng.integers(k - 1)) % k)
            recs.append(W.gate(name, t, control=c, angle=float(rng.uniform(0, 2 * np.pi))))
        elif name == "U":
            recs.append(W.gate("U", t, u=W.random_unitaries(int(rng.integers(1 << 30)), 1)[0]))
        else:
            recs.append(W.gate(name, t, angle=float(rng.uniform(0, 2 * np.pi))))
    gates = np.concatenate(recs)
    # the block's 32 x 32 unitary: its columns are the engine's images of the basis states
    cols = []
    for b in range(1 << k):
        sv = capi.Statevector(k)
        sv.set_basis(b)
        sv.apply(gates)
        cols.append(sv.download())
        sv.close()
    U = np.stack(cols, axis=1)
    # real form of y = U x on interleaved (re, im) pairs: yr = xr @ Mr
    Mr = np.zeros((2 << k, 2 << k))
    Mr[0::2, 0::2] = U.real.T
    Mr[1::2, 0::2] = -U.imag.T
    Mr[0::2, 1::2] = U.imag.T
    Mr[1::2, 1::2] = U.real.T
    N2 = 2 << n
    init = W.random_layers(n, 1, seed=17, mixed=True)
    want = capi.Statevector(n)
    want.apply(init)
    want.apply(gates)
    tw = torch.as_tensor(_DeviceArray(want.device_ptr(), N2, "<f8"), device="cuda")
    s64 = capi.Statevector(n, capi.KT_C64)
    t64 = torch.as_tensor(_DeviceArray(s64.device_ptr(), N2, "<f4"), device="cuda")
    stream = torch.cuda.current_stream()

    def timed(fn):
        best = None
        for _ in range(1 + reps):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) / 1e3
            best = t if best is None else min(best, t)
        return best

    def max_err(x):
        worst = 0.0
        chunk = 1 << 26
        for a in range(0, N2, chunk):
            worst = max(worst, float((tw[a:a + chunk] - x[a:a + chunk].double()).abs().max()))
        return worst

    s64.set_basis(0)
    s64.apply(init)
    x0 = t64.clone()
    s64.prepare(gates)

    def eng():
        t64.copy_(x0)
        s64.apply(gates)

    copy_t = timed(lambda: t64.copy_(x0))
    t_eng = timed(eng) - copy_t
    err_eng = max_err(t64)
    tc = {}
    for name, passes in (("tcgen05_4xtf32", 4), ("tcgen05_3xtf32", 3), ("tcgen05_tf32", 1)):
        def run_tc(p=passes):
            t64.copy_(x0)
            s64.apply_dense5(U, p)
        t = timed(run_tc) - copy_t
        tc[name] = {"seconds": t, "max_abs_error": max_err(t64)}
    xr = x0.view(-1, 2 << k)
    y = torch.empty_like(xr)
    m32 = torch.as_tensor(Mr, dtype=torch.float32, device="cuda")
    out = {"qubits": n, "block_qubits": k, "gates": int(gates.size), "state_bytes": 4 * N2,
           "engine": {"seconds": t_eng, "max_abs_error": err_eng}, **tc}
    for name, tf32 in (("gemm_fp32", False), ("gemm_tf32", True)):
        torch.backends.cuda.matmul.allow_tf32 = tf32
        t = timed(lambda: torch.matmul(xr, m32, out=y))
        out[name] = {"seconds": t, "max_abs_error": max_err(y.view(-1))}
    torch.backends.cuda.matmul.allow_tf32 = False
    for key in ("engine", "tcgen05_4xtf32", "tcgen05_3xtf32", "tcgen05_tf32", "gemm_fp32", "gemm_tf32"):
        out[key]["alg_gbs"] = 2 * 4 * N2 / out[key]["seconds"] / 1e9
    print(json.dumps(out))
    s64.close()
    want.close()


CASES = {k[5:]: v for k, v in globals().items() if k.startswith("case_")}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("case", choices=sorted(CASES))
    ap.add_argument("--qubits", type=int, default=26, help="state size (density matrices use half)")
    ap.add_argument("--reps", type=int, default=2, help="runs after the warm-up run")
    args = ap.parse_args(argv)
    CASES[args.case](args.qubits, args.reps)
    print(f"profile case {args.case} done ({args.qubits} qubits, 1 + {args.reps} runs)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
