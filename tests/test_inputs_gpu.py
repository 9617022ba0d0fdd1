"""The device path against the reference on the reference's own input files
(tests/golden/inputs): real molecules with cusp replacement, Cambridge
three-body Jastrows, several determinants, a 70-electron system whose
spins keep their inverses in HBM."""
import numpy as np
import pytest

from inputs_common import INPUT_CASES, load_input_case, replay_against_reference
from qmcbeaver_b200.api import QMCB200Functions

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", INPUT_CASES)
def test_gpu_reproduces_reference_inputs(case):
    s, d = load_input_case(case)
    W = d["R"].shape[1]
    f = QMCB200Functions(s, W, qf_modification=int(d["qf_mod"]), dt=float(d["dt"]))
    slots = np.arange(W)
    replay_against_reference(s, d, lambda e, R: f.evaluate(slots, R, e), f"gpu/{case}")
    f.close()
