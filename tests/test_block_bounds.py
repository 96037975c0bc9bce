"""The per-block bound tool on a synthetic launch list (CPU): the CSV
parser's units, the cut into applies, and the bounds' arithmetic."""
import csv

import numpy as np

from kettle_b200 import block_bounds as BB
from kettle_b200 import capi
from kettle_b200 import workloads as W


def _write(path, rows):
    with open(path, "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(["ID", "Kernel Name", "Metric Name", "Metric Unit", "Metric Value"])
        for i, (name, unit, value) in enumerate(rows):
            w.writerow([i, name, "gpu__time_duration.sum", unit, value])


def test_launch_times_units(tmp_path):
    p = tmp_path / "l.csv"
    _write(p, [("kt_jb0", "msecond", "1.5"), ("k_set_basis<double2>", "usecond", "250"), ("kt_jb1", "nsecond", "2,000,000")])
    t = BB.launch_times(str(p))
    assert [k for k, _ in t] == ["kt_jb0", "k_set_basis<double2>", "kt_jb1"]
    assert np.allclose([v for _, v in t], [1.5, 0.25, 2.0])


def test_bounds_table(tmp_path, capsys):
    n, layers = 14, 3
    pb = capi.plan_blocks(n, W.random_layers(n, layers, seed=5, mixed=True))
    rows = []
    for _ in range(2):  # two applies
        rows.append(("k_set_basis<double2>", "usecond", "10"))
        rows += [(f"kt_jb{b}", "msecond", str(1.0 + b)) for b in range(len(pb))]
    p = tmp_path / "l.csv"
    _write(p, rows)
    assert BB.main([str(p), "--qubits", str(n), "--layers", str(layers), "--seed", "5", "--clock-mhz", "1965",
                    "--hbm-gbs", "6550.7"]) == 0
    out = capsys.readouterr().out
    assert f"{len(pb)} blocks, 2 applies" in out
    assert out.count("\n| ") == len(pb) + 1  # header and one row per block
