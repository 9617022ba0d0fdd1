"""Serving loop: jobs admitted by device footprint, run concurrently (one
stream per job, or all active jobs stepped together as one group), each
job's energies the same alone and in the mix."""
import numpy as np
import pytest

from qmcbeaver_b200.serving import Job, Server, blocked_error, make_jobs, state_footprint

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["streams", "group"])
def test_jobs_complete_and_report_latency(mode):
    jobs = make_jobs(6, rate=50.0, seed=3, electrons=(4, 20), walkers=(256, 512), target_error=0.5, max_sweeps=40)
    out = Server(max_active=4, mode=mode, batch_steps=24).run(jobs)
    assert out["jobs"] == 6
    assert out["latency_p50_s"] is not None and out["latency_p99_s"] >= out["latency_p50_s"]
    for j in jobs:
        assert j.finished is not None and np.isfinite(j.energy)
        assert len(j.energies) >= j.min_blocks


@pytest.mark.parametrize("mode", ["streams", "group"])
def test_result_same_alone_and_in_mix(mode):
    def fresh():
        js = make_jobs(5, rate=1e3, seed=5, electrons=(6, 16), walkers=(256, 512), target_error=0.0, max_sweeps=24)
        for j in js:
            j.arrival = 0.0
        return js
    mix = fresh()
    Server(max_active=5, mode=mode, batch_steps=16).run(mix)
    alone = fresh()[2]
    Server(max_active=1, mode=mode, batch_steps=16).run([alone])
    assert len(alone.energies) == len(mix[2].energies) == 24
    np.testing.assert_allclose(alone.energies, mix[2].energies, rtol=1e-10, atol=0)


def test_admission_respects_footprint_budget():
    jobs = make_jobs(4, rate=1e3, seed=7, electrons=(10, 10), walkers=(512, 512), target_error=0.0, max_sweeps=4)
    need = state_footprint(jobs[0].system, 512)
    srv = Server(hbm_budget=int(need * 1.5), max_active=8)   # room for one job at a time
    out = srv.run(jobs)
    assert out["jobs"] == 4
    # with room for one job only, each job is admitted after the previous finished
    order = sorted(jobs, key=lambda j: j.admitted)
    for a, b in zip(order, order[1:]):
        assert b.admitted >= a.finished - 1e-6


def test_footprint_matches_library():
    from qmcbeaver_b200.api import QMCB200Functions
    from qmcbeaver_b200.system import make_system
    from qmcbeaver_b200.system import make_random_molecule
    from qmcbeaver_b200.desc import QMCB_PREC_BF16X3_TC, QMCB_PREC_FP64, QMCB_PREC_INT8_SLICES
    for s in (make_system("vmc_water_10e"), make_system("dmc_6nuc_30e"),
              make_random_molecule(60, 8, 120, 8.0, (1, 6, 7, 8), seed=2)):
        for prec in (QMCB_PREC_FP64, QMCB_PREC_INT8_SLICES, QMCB_PREC_BF16X3_TC):
            f = QMCB200Functions(s, 2 * 300, precision=prec)
            assert f.state_bytes() == state_footprint(s, 300, prec), prec
            f.close()


def test_tensor_core_rows_jobs_same_alone_and_in_mix():
    """Jobs on split-BF16 tensor-core rows next to FP64 jobs: each job's
    energies are the same alone and in the mix."""
    from qmcbeaver_b200.desc import QMCB_PREC_BF16X3_TC

    def fresh():
        js = make_jobs(4, rate=1e3, seed=9, electrons=(6, 40), walkers=(256, 512), target_error=0.0, max_sweeps=16)
        for k, j in enumerate(js):
            j.arrival = 0.0
            if k % 2 == 0:
                j.precision = QMCB_PREC_BF16X3_TC
        return js
    mix = fresh()
    Server(max_active=4, mode="streams").run(mix)
    for k in (0, 1):
        alone = fresh()[k]
        Server(max_active=1, mode="streams").run([alone])
        assert len(alone.energies) == len(mix[k].energies) == 16
        np.testing.assert_allclose(alone.energies, mix[k].energies, rtol=1e-10, atol=0)
