"""Drop-in check: tests/cpp/dropin_main.cpp uses only the kettle C++ API.
Built against the reference (oracle/_ref/dropin_ref, from the reference's own
sources) and against this engine's ket:: front end (kettle_b200/lib/dropin_b200),
both binaries must print the same results: amplitudes, expectation value and
density matrix within 1e-12, sampled counts and measured bits identical, and
for a circuit with mid-circuit measurements, if / if-else statements and
circuit loggers: the same measured bits, logged registers and states; and
for the on-disk formats: the same statevector text byte for byte, the same
states read back from statevector and numpy text, the same Hamiltonian read
from Pauli-operator text, and the same reader errors."""
import pathlib
import subprocess

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
REF_BIN = ROOT / "oracle" / "_ref" / "dropin_ref"
OUR_BIN = ROOT / "kettle_b200" / "lib" / "dropin_b200"

pytestmark = pytest.mark.gpu


def _run(exe, *args):
    out = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    rec = {"amp": {}, "mamp": {}, "cfamp": {}, "ioamp": {}, "npamp": {}, "rho": {}, "count": {}, "expect": None,
           "cbits": None, "cfbits": None, "logbit": {}, "logamp": {}, "svtext": {}, "svload": {}, "ioerr": {},
           "cgamp": {}, "ptrace": {}, "tensor": {}, "nq": {}, "tpamp": {}, "psamp": {}, "svtp": {}, "pmem": {},
           "pcraw": {}, "pcmarg": {}, "pcodd": {}, "ccmarg": {}, "dmmrho": {}}
    for line in out.stdout.splitlines():
        f = line.split()
        if f[0] in ("amp", "mamp", "cfamp", "ioamp", "npamp", "cgamp", "tpamp", "psamp", "svtp"):
            rec[f[0]][int(f[1])] = complex(float(f[2]), float(f[3]))
        elif f[0] == "cfbits":
            rec["cfbits"] = tuple(int(x) for x in f[1:])
        elif f[0] == "logbit":
            rec["logbit"][(int(f[1]), int(f[2]))] = int(f[3])
        elif f[0] == "logamp":
            rec["logamp"][(int(f[1]), int(f[2]))] = complex(float(f[3]), float(f[4]))
        elif f[0] == "rho":
            rec["rho"][(int(f[1]), int(f[2]))] = complex(float(f[3]), float(f[4]))
        elif f[0] == "count":
            rec["count"][f[1]] = int(f[2])
        elif f[0] == "expect":
            rec["expect"] = complex(float(f[1]), float(f[2]))
        elif f[0] == "svtext":
            rec["svtext"][int(f[1])] = (int(f[2]), f[3])
        elif f[0] == "svload":
            rec["svload"][int(f[1])] = (int(f[2]), float(f[3]))
        elif f[0] in ("npfile",):
            rec[f[0]] = float(f[1])
        elif f[0] in ("pauliop",):
            rec[f[0]] = (int(f[1]), complex(float(f[2]), float(f[3])))
        elif f[0] in ("pauliopfile",):
            rec[f[0]] = complex(float(f[1]), float(f[2]))
        elif f[0] in ("ptrace", "tensor") and f[2] == "nq":
            rec["nq"][(f[0], int(f[1]))] = int(f[3])
        elif f[0] in ("ptrace", "tensor"):
            rec[f[0]][(int(f[1]), int(f[2]), int(f[3]))] = complex(float(f[4]), float(f[5]))
        elif f[0] == "tpgate":
            rec.setdefault("tpgate", []).append((int(f[2]), int(f[3]), int(f[4]), float(f[5])))
        elif f[0] == "tpelems":
            rec[f[0]] = tuple(int(x) for x in f[1:])
        elif f[0] == "tperr":
            rec[f[0]] = f[1]
        elif f[0] in ("cgelems", "pterr"):
            rec[f[0]] = int(f[1])
        elif f[0] == "sqrtu":
            rec[f[0]] = np.array([float(x) for x in f[1:]])
        elif f[0] == "purity":
            rec[f[0]] = (complex(float(f[1]), float(f[2])), int(f[3]), complex(float(f[4]), float(f[5])), int(f[6]))
        elif f[0] == "ioerr":
            rec["ioerr"][f[1]] = f[2]
        elif f[0] == "cbit0":
            rec["cbits"] = (int(f[1]), int(f[3]))
        elif f[0] in ("pmem", "pcraw", "pcodd"):
            rec[f[0]][int(f[1])] = int(f[2])
        elif f[0] in ("pcmarg", "ccmarg"):
            rec[f[0]][f[1]] = int(f[2])
        elif f[0] == "diagexp":
            rec[f[0]] = complex(float(f[1]), float(f[2]))
        elif f[0] in ("pserr", "pmerr"):
            rec[f[0]] = int(f[1])
        elif f[0] == "dmmbits":
            rec[f[0]] = tuple(int(x) for x in f[1:])
        elif f[0] == "dmmrho":
            rec[f[0]][(int(f[1]), int(f[2]))] = complex(float(f[3]), float(f[4]))
    return rec


@pytest.mark.parametrize("n,layers,seed", [(6, 4, 1), (11, 6, 2), (14, 3, 3)])
def test_dropin_same_results(engine, n, layers, seed):
    if not REF_BIN.exists():
        pytest.skip("reference build of the drop-in program is absent")
    assert OUR_BIN.exists(), "engine build of the drop-in program is missing"
    ref = _run(REF_BIN, n, layers, seed)
    our = _run(OUR_BIN, n, layers, seed)
    a = np.array([ref["amp"][i] for i in sorted(ref["amp"])])
    b = np.array([our["amp"][i] for i in sorted(our["amp"])])
    assert np.abs(a - b).max() < 1e-12
    assert abs(ref["expect"] - our["expect"]) < 1e-12
    assert ref["count"] == our["count"]
    assert ref["cbits"] == our["cbits"]
    ma = np.array([ref["mamp"][i] for i in sorted(ref["mamp"])])
    mb = np.array([our["mamp"][i] for i in sorted(our["mamp"])])
    assert np.abs(ma - mb).max() < 1e-12
    # classical control flow and circuit loggers
    assert ref["cfbits"] == our["cfbits"]
    assert ref["logbit"] == our["logbit"] and len(ref["logbit"]) == 2 * n
    assert sorted(ref["logamp"]) == sorted(our["logamp"]) and len(ref["logamp"]) == 1 << n
    la = np.array([ref["logamp"][k] for k in sorted(ref["logamp"])])
    lb = np.array([our["logamp"][k] for k in sorted(our["logamp"])])
    assert np.abs(la - lb).max() < 1e-12
    ca = np.array([ref["cfamp"][i] for i in sorted(ref["cfamp"])])
    cb = np.array([our["cfamp"][i] for i in sorted(our["cfamp"])])
    assert np.abs(ca - cb).max() < 1e-12
    ra = np.array([ref["rho"][k] for k in sorted(ref["rho"])])
    rb = np.array([our["rho"][k] for k in sorted(our["rho"])])
    assert np.abs(ra - rb).max() < 1e-12
    # on-disk formats: the statevector text is the same bytes in both endians
    assert ref["svtext"] == our["svtext"] and len(our["svtext"]) == 2
    for endian in (0, 1):
        assert our["svload"][endian][0] == n and our["svload"][endian][1] < 1e-14
    ia = np.array([ref["ioamp"][i] for i in sorted(ref["ioamp"])])
    ib = np.array([our["ioamp"][i] for i in sorted(our["ioamp"])])
    assert ia.size == b.size and np.abs(ia - ib).max() < 1e-12
    assert np.abs(ib - b).max() < 1e-13    # 14 printed digits
    na = np.array([ref["npamp"][i] for i in sorted(ref["npamp"])])
    nb = np.array([our["npamp"][i] for i in sorted(our["npamp"])])
    flip = [int(format(i, f"0{n}b")[::-1], 2) for i in range(1 << n)]
    assert np.abs(na - nb).max() < 1e-12
    assert np.abs(nb - b[flip]).max() < 1e-7   # every third value has 9 significant digits
    assert our["npfile"] < 1e-7
    assert ref["pauliop"][0] == our["pauliop"][0] == 30
    assert abs(ref["pauliop"][1] - our["pauliop"][1]) < 1e-12
    assert abs(our["pauliopfile"] - our["pauliop"][1]) == 0.0
    assert ref["ioerr"] == our["ioerr"] == {"load": "1", "numpy": "1", "pauli": "1", "badterm": "out_of_range"}
    # compound gates
    if n >= 4:
        assert ref["cgelems"] == our["cgelems"]
        ga = np.array([ref["cgamp"][i] for i in sorted(ref["cgamp"])])
        gb = np.array([our["cgamp"][i] for i in sorted(our["cgamp"])])
        assert ga.size == 1 << n and np.abs(ga - gb).max() < 1e-12
        assert np.abs(ref["sqrtu"] - our["sqrtu"]).max() < 1e-14
    # density-matrix partial traces, tensor products, purity
    assert ref["nq"] == our["nq"]
    for key in ("ptrace", "tensor"):
        assert sorted(ref[key]) == sorted(our[key]) and len(ref[key]) > 0
        pa = np.array([ref[key][k] for k in sorted(ref[key])])
        pb = np.array([our[key][k] for k in sorted(our[key])])
        assert np.abs(pa - pb).max() < 1e-12
    assert ref["pterr"] == our["pterr"] == 1
    rp, op = ref["purity"], our["purity"]
    assert abs(rp[0] - op[0]) < 1e-12 and abs(rp[2] - op[2]) < 1e-12
    assert rp[1] == op[1] and rp[3] == op[3]
    # circuit transforms
    ta, tb = ref["tpgate"], our["tpgate"]
    assert len(ta) == len(tb) == our["tpelems"][1]
    for x, y in zip(ta, tb):
        assert x[:3] == y[:3] and abs(x[3] - y[3]) < 1e-12
    assert ref["tpelems"] == our["tpelems"]
    pa = np.array([ref["tpamp"][i] for i in sorted(ref["tpamp"])])
    pb = np.array([our["tpamp"][i] for i in sorted(our["tpamp"])])
    assert pa.size == 1 << n and np.abs(pa - pb).max() < 1e-12
    assert ref["tperr"] == our["tperr"] == "qubits"
    # Pauli string on a state, statevector tensor product, diagonal expectation,
    # probability-vector sampling, circuit-and-state marginal counts, M on a density matrix
    for key, size in (("psamp", 1 << n), ("svtp", 1 << (n + 1))):
        pa = np.array([ref[key][i] for i in sorted(ref[key])])
        pb = np.array([our[key][i] for i in sorted(our[key])])
        assert pa.size == size and np.abs(pa - pb).max() < 1e-12, key
    assert ref["pserr"] == our["pserr"] == 1
    assert abs(ref["diagexp"] - our["diagexp"]) < 1e-12
    for key in ("pmem", "pcraw", "pcmarg", "pcodd", "ccmarg"):
        assert ref[key] == our[key] and len(ref[key]) > 0, key
    assert ref["pmerr"] == our["pmerr"] == 1
    assert ref["dmmbits"] == our["dmmbits"]
    da = np.array([ref["dmmrho"][k] for k in sorted(ref["dmmrho"])])
    db = np.array([our["dmmrho"][k] for k in sorted(our["dmmrho"])])
    assert da.size == 4 ** min(n, 5) and np.abs(da - db).max() < 1e-12
