"""The oracle against the reference on the reference's own input files
(real molecules with cusp replacement, three-body Jastrows and several
determinants): the fixtures of tests/golden/inputs."""
import pytest

from inputs_common import INPUT_CASES, load_input_case, replay_against_reference


def test_input_cases_present():
    assert {"h2o", "oepi", "chkpnt", "det", "be_mcscf", "ne0p", "annulene", "hmx"} <= set(INPUT_CASES)


@pytest.mark.parametrize("case", INPUT_CASES)
def test_oracle_reproduces_reference_inputs(case):
    from oracle.evaluators import OracleEvaluator
    s, d = load_input_case(case)
    ev = OracleEvaluator(s, qf_mod=int(d["qf_mod"]), dt=float(d["dt"]))
    ws = ev.new_walkers(d["R"].shape[1])

    def run(e, R):
        ev.evaluate(ws, R, e)
        return ev.results(ws)

    replay_against_reference(s, d, run, f"oracle/{case}")
