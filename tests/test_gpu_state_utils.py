"""The state part of the host-utility drop-in check on a GPU: seeded random
states, projections of them and the io/ text formats (statevector save and
load, numpy text, Pauli-operator text) through the engine (states in GPU
memory),
against the reference build of tests/cpp/dropin_host_main.cpp, text for text
(doubles in hexadecimal: bit for bit).  The CPU suite runs the same program
over host-memory stand-ins of the state calls (tests/test_dropin_host.py)."""
import pytest

from test_dropin_host import OUR_BIN, _diff, _ref, _run

pytestmark = pytest.mark.gpu


def test_state_utilities_match_reference_on_gpu(engine):
    want = _ref("states")
    assert OUR_BIN.exists(), "front-end build of the host-utility program missing (kettle_b200.build)"
    got = _run(OUR_BIN, "states")
    assert got == want, _diff(want, got)
