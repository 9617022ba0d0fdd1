"""Groups (qmcb_group_*): the walkers of several systems of different sizes
stepped by one persistent launch per bucket.  Each member must follow
exactly the chain it follows when its own handle steps it (same random
streams, same arithmetic), whatever launch configuration the tuner tries."""
import numpy as np
import pytest

from qmcbeaver_b200.api import QMCB200Functions, QMCB200Group, QMCBError
from qmcbeaver_b200.desc import (QMCB_DMC, QMCB_ECUT_BDJM_PUSH88, QMCB_EMOD_UMRIGAR93, QMCB_IMPORTANCE_SAMPLING,
                                 QMCB_PREC_MIXED, QMCB_QF_UMRIGAR93_UNEQUAL, QMCB_UMRIGAR93_IMPORTANCE_SAMPLING,
                                 run_params)
from qmcbeaver_b200.system import make_random_molecule, with_determinants, with_three_body

pytestmark = pytest.mark.gpu

# (electrons, nuclei, basis functions, walkers): uneven sizes, as in a
# batch of serving jobs
SIZES = [(4, 1, 16, 300), (30, 6, 120, 700), (10, 2, 40, 513), (56, 10, 224, 260), (18, 3, 72, 900)]


def _systems(extra_threebody=False):
    out = []
    for k, (ne, nn, nb, w) in enumerate(SIZES):
        s = make_random_molecule(ne, nn, nb, 5.0 + ne / 10, (1, 6, 7, 8), seed=10 + k)
        if extra_threebody and k == 2:
            s = with_three_body(s, seed=3)
        if extra_threebody and k == 4:
            s = with_determinants(s, 6, 3, seed=2)  # several determinants
        out.append((s, w))
    return out


def _params(k, sampling=QMCB_IMPORTANCE_SAMPLING):
    return run_params(sampling=sampling, qf_modification=QMCB_QF_UMRIGAR93_UNEQUAL, dt=0.01, seed=100 + k,
                      rel_cutoff=0.0)


def _dmc_params(k, e0):
    # DMC with the Umrigar93 energy modification and the BDJM cutoff around
    # the initial mean local energy, a full refresh every 25 steps (so the
    # group takes its launch-by-launch path, not the graph)
    return run_params(run_type=QMCB_DMC, sampling=QMCB_IMPORTANCE_SAMPLING, qf_modification=QMCB_QF_UMRIGAR93_UNEQUAL,
                      energy_modification=QMCB_EMOD_UMRIGAR93, energy_cutoff=QMCB_ECUT_BDJM_PUSH88, dt=0.01,
                      refresh_interval=25, energy_trial=e0, energy_estimated=e0, energy_original=e0,
                      population_control=100.0, seed=200 + k, rel_cutoff=0.0)


def _handles(systems, params):
    hs = []
    for k, (s, w) in enumerate(systems):
        f = QMCB200Functions(s, 2 * w, params(k))
        f.init_walkers(s.initial_positions(w, seed=k + 1))
        hs.append(f)
    return hs


def _first_steps(systems):
    # members start at different points of their own step sequences
    return [3 * k + 1 for k in range(len(systems))]


@pytest.mark.parametrize("extras", [False, True])
def test_vmc_group_matches_members_alone(extras):
    systems = _systems(extra_threebody=extras)
    sampling = QMCB_UMRIGAR93_IMPORTANCE_SAMPLING if extras else QMCB_IMPORTANCE_SAMPLING

    def params(k):
        return _params(k, sampling=sampling if k in (0, 2) else QMCB_IMPORTANCE_SAMPLING)

    solo, grouped = _handles(systems, params), _handles(systems, params)
    g = QMCB200Group(grouped)
    fs = _first_steps(systems)
    n_batches, n_steps = 7, 13
    cfg = g.config()
    assert cfg["n_configs"] >= 2
    for b in range(n_batches):
        st_g = g.run_steps([f + b * n_steps for f in fs], n_steps)
        for k, f in enumerate(solo):
            st = f.run_steps(fs[k] + b * n_steps, n_steps)
            assert st.n_moves == st_g[k].n_moves
            assert st_g[k].sum_weight_energy == pytest.approx(st.sum_weight_energy, rel=1e-12, abs=1e-9)
            assert st_g[k].sum_accept == pytest.approx(st.sum_accept, rel=1e-12)
    # every candidate configuration was timed, the fastest kept
    cfg = g.config()
    assert cfg["chosen"] >= 0 and cfg["last"] == cfg["chosen"]
    for a, b in zip(solo, grouped):
        wa, wb = a.get_walkers(), b.get_walkers()
        assert np.array_equal(wa["R"], wb["R"])
        assert np.allclose(wa["e_local"], wb["e_local"], rtol=1e-12, atol=1e-12)


def test_group_members_on_tensor_core_rows_match_members_alone():
    """Members whose orbital rows come from the batched tensor-core
    contraction (int8 digit planes at FP64 accuracy, BF16 and split BF16 with
    FP32 accumulation) next to FP64 members, all refreshing their inverses in
    FP64 every 7 steps: the group launches each rows member's prep and
    contraction before the persistent move kernel, and every member follows
    exactly its own handle's chain."""
    from qmcbeaver_b200.desc import QMCB_PREC_BF16_TC, QMCB_PREC_BF16X3_TC, QMCB_PREC_FP64, QMCB_PREC_INT8_SLICES
    systems = _systems()
    precs = [QMCB_PREC_BF16X3_TC, QMCB_PREC_INT8_SLICES, QMCB_PREC_FP64, QMCB_PREC_BF16_TC, QMCB_PREC_INT8_SLICES]

    def params(k):
        p = _params(k)
        p.precision = precs[k]
        p.refresh_interval = 7  # FP64 refreshes of the inverses inside the group's batches
        return p

    solo, grouped = _handles(systems, params), _handles(systems, params)
    g = QMCB200Group(grouped)
    fs = _first_steps(systems)
    n_steps = 11
    for b in range(4):
        st_g = g.run_steps([f + b * n_steps for f in fs], n_steps)
        for k, f in enumerate(solo):
            st = f.run_steps(fs[k] + b * n_steps, n_steps)
            assert st.n_moves == st_g[k].n_moves
            assert st_g[k].sum_accept == pytest.approx(st.sum_accept, rel=1e-12)
    for a, b in zip(solo, grouped):
        wa, wb = a.get_walkers(), b.get_walkers()
        assert np.isfinite(wa["R"]).all()
        assert np.array_equal(wa["R"], wb["R"])
        assert np.allclose(wa["e_local"], wb["e_local"], rtol=1e-12, atol=1e-12)
    g.close()


def test_every_configuration_gives_the_same_chain():
    systems = _systems()
    ref = _handles(systems, _params)
    fs = _first_steps(systems)
    for k, f in enumerate(ref):
        f.run_steps(fs[k], 20)
    want = [f.get_walkers()["R"] for f in ref]
    probe = _handles(systems, _params)
    n = QMCB200Group(probe).config()["n_configs"]
    for c in range(n):
        hs = _handles(systems, _params)
        g = QMCB200Group(hs)
        g.set_config(c)
        g.run_steps(fs, 20)
        assert g.config()["last"] == c
        for w, h in zip(want, hs):
            assert np.array_equal(w, h.get_walkers()["R"])


def test_dmc_group_branches_like_members_alone():
    systems = _systems()
    e0 = []
    for k, f in enumerate(_handles(systems, _params)):
        e0.append(float(np.median(f.get_walkers()["e_local"])))

    def params(k):
        return _dmc_params(k, e0[k])

    solo, grouped = _handles(systems, params), _handles(systems, params)
    g = QMCB200Group(grouped)
    fs = [0] * len(systems)
    # two batches: every member branches at least once (steps that move
    # electron 0); the trial energies feed back through device sums
    for b in range(2):
        n_steps = 60
        st_g = g.run_steps([f + b * n_steps for f in fs], n_steps)
        for k, f in enumerate(solo):
            st = f.run_steps(fs[k] + b * n_steps, n_steps)
            assert st_g[k].n_walkers == st.n_walkers
            assert st_g[k].final_weight == pytest.approx(st.final_weight, rel=1e-9)
            assert st_g[k].sum_weight_energy == pytest.approx(st.sum_weight_energy, rel=1e-9)
    for a, b in zip(solo, grouped):
        wa, wb = a.get_walkers(), b.get_walkers()
        assert np.array_equal(wa["R"], wb["R"])
        assert np.allclose(wa["weight"], wb["weight"], rtol=1e-9)


def test_group_refuses_unsupported_members():
    s = make_random_molecule(8, 2, 32, 5.0, (1, 6, 7, 8), seed=4)
    a = QMCB200Functions(s, 64, _params(0))
    c = QMCB200Functions(s, 64, run_params(precision=QMCB_PREC_MIXED, dt=0.01))
    c.init_walkers(s.initial_positions(32, seed=1))
    a.init_walkers(s.initial_positions(32, seed=2))
    g = QMCB200Group([a, c])
    with pytest.raises(QMCBError, match="FP64"):
        g.run_steps(0, 4)


def test_group_members_match_the_oracle():
    """Each member of a group, after a batch of group steps, holds the local
    energy and log|psi| the oracle computes from scratch at the member's
    current positions (to the drift of the Sherman-Morrison chain, 1e-8
    relative, as for a single handle), on walkers whose Slater matrices are
    well conditioned."""
    from helpers import cond_bounds, slater_conditions
    from oracle.evaluators import OracleEvaluator
    systems = _systems(extra_threebody=True)
    hs = _handles(systems, _params)
    g = QMCB200Group(hs)
    g.run_steps(_first_steps(systems), 40)
    g.close()
    for (s, w), f in zip(systems, hs):
        got = f.get_walkers()
        n = min(64, len(got["weight"]))
        orc = OracleEvaluator(s, qf_mod=QMCB_QF_UMRIGAR93_UNEQUAL, dt=0.01)
        ws = orc.new_walkers(n)
        orc.evaluate(ws, got["R"][:n], -1)
        ref = orc.results(ws)
        ok = (ref["singular"] == 0) & (slater_conditions(orc, ws, s) < cond_bounds(s)[1])
        assert ok.sum() >= n // 4, (s.name, ok.sum())
        kap = np.maximum(np.asarray(orc.kappa(ws), np.float64), 1.0)  # several determinants' mixing
        for k in ("e_local", "log_abs_psi"):
            err = np.abs(got[k][:n] - ref[k]) / np.maximum(np.abs(ref[k]), 1.0) / kap
            assert np.max(err[ok]) < 1e-8, (s.name, k, float(np.max(err[ok])))
        f.close()
