"""Per-block bounds of a fused apply against measured per-block times.

    python -m kettle_b200.block_bounds <launch-list.csv> [--qubits 30] [--layers 40]
        [--seed 2024] [--clock-mhz 1880] [--hbm-gbs G]

The launch list is an Nsight Compute CSV with `gpu__time_duration.sum` per
launch (`ncu --metrics gpu__time_duration.sum --csv --log-file ...`) of runs
that apply the benchmark circuit (`workloads.random_layers(qubits, layers,
seed, mixed=True)`, complex128).  Its `kt_jb*` launches are cut into whole
applies of the planned block count and each block's median is set beside
three bounds of that block, all per pass over the 2^n amplitudes:

  t_dram = 2 x 16 B x 2^n / HBM bandwidth            (read and write the state once)
  t_fp64 = FP64 operations per amplitude x 2^n / (SMs x 64 per clock x clock)
  t_smem = transposes x 2 x 16 B x 2^n / (SMs x 128 B per clock x clock)

The operation and transpose counts are the planner's own (`kt_plan_blocks`,
no GPU needed).  The HBM figure defaults to `hbm_gbs` of MEASURED_PEAKS.json
at the repository root when that file exists, else 6650 GB/s.  Prints a
markdown table of every block and a least-squares fit of the measured times
to a + b t_fp64 + c t_smem.
"""
from __future__ import annotations

import argparse
import csv
import json
import pathlib
import sys

import numpy as np

from . import capi
from . import workloads as W

SMS = 148


def launch_times(path: str) -> list[tuple[str, float]]:
    """(kernel name, milliseconds) of every launch in an ncu CSV launch list."""
    rows = list(csv.reader(open(path)))
    hi = next(i for i, r in enumerate(rows) if "Kernel Name" in r)
    h = rows[hi]
    ki, mi, vi = h.index("Kernel Name"), h.index("Metric Name"), h.index("Metric Value")
    ui = h.index("Metric Unit") if "Metric Unit" in h else None
    scale = {"nsecond": 1e-6, "ns": 1e-6, "usecond": 1e-3, "us": 1e-3, "msecond": 1.0, "ms": 1.0}
    out = []
    for r in rows[hi + 1:]:
        if len(r) > vi and r[mi] == "gpu__time_duration.sum":
            u = r[ui] if ui is not None else "nsecond"
            out.append((r[ki], float(r[vi].replace(",", "")) * scale.get(u, 1e-6)))
    return out


def default_hbm() -> float:
    p = pathlib.Path(__file__).resolve().parent.parent / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("launches")
    ap.add_argument("--qubits", type=int, default=30)
    ap.add_argument("--layers", type=int, default=40)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--clock-mhz", type=float, default=1880.0, help="SM clock the launch list ran at")
    ap.add_argument("--hbm-gbs", type=float, default=None)
    a = ap.parse_args(argv)
    hbm = (a.hbm_gbs or default_hbm()) * 1e9
    clk = a.clock_mhz * 1e6
    pb = capi.plan_blocks(a.qubits, W.random_layers(a.qubits, a.layers, seed=a.seed, mixed=True))
    nb = len(pb)
    jb = [t for k, t in launch_times(a.launches) if k.startswith("kt_jb")]
    applies = len(jb) // nb
    if applies == 0:
        print(f"the launch list holds {len(jb)} kt_jb launches, fewer than one apply of {nb} blocks")
        return 1
    meas = np.median(np.array([jb[s * nb:(s + 1) * nb] for s in range(applies)]), axis=0)
    amps = 2.0 ** a.qubits
    t_dram = 2 * 16 * amps / hbm * 1e3
    t_fp = pb[:, 3] * amps / (SMS * 64 * clk) * 1e3
    t_sm = pb[:, 2] * 32 * amps / (SMS * 128 * clk) * 1e3
    bound = np.maximum(t_dram, np.maximum(t_fp, t_sm))
    print(f"{nb} blocks, {applies} applies in the list (median per block), clock {a.clock_mhz:.0f} MHz, "
          f"HBM {hbm / 1e9:.1f} GB/s, t_dram {t_dram:.2f} ms per block\n")
    print("| block | ops | phases | transposes | FP64 / amplitude | t_fp64 (ms) | t_smem (ms) | max bound (ms) "
          "| t_fp64 + t_smem (ms) | measured (ms) | measured / max bound |")
    print("|---:|---:|---:|---:|---:|---:|---:|---:|---:|---:|---:|")
    for b in range(nb):
        print(f"| {b} | {int(pb[b, 0])} | {int(pb[b, 1])} | {int(pb[b, 2])} | {pb[b, 3]:.1f} | {t_fp[b]:.2f} | "
              f"{t_sm[b]:.2f} | {bound[b]:.2f} | {t_fp[b] + t_sm[b]:.2f} | {meas[b]:.2f} | {meas[b] / bound[b]:.2f} |")
    print(f"\nsum over blocks: measured {meas.sum():.1f} ms, max bounds {bound.sum():.1f} ms, "
          f"DRAM alone {nb * t_dram:.1f} ms, FP64 {t_fp.sum():.1f} ms, transposes {t_sm.sum():.1f} ms")
    A = np.vstack([np.ones(nb), t_fp, t_sm]).T
    coef, *_ = np.linalg.lstsq(A, meas, rcond=None)
    r = np.corrcoef(meas, t_fp + t_sm)[0, 1]
    print(f"least squares: measured = {coef[0]:.2f} ms + {coef[1]:.3f} t_fp64 + {coef[2]:.3f} t_smem; "
          f"correlation of measured with t_fp64 + t_smem {r:.3f}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
