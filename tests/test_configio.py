"""Configuration files (.cfgs): the reader / writer in
qmcbeaver_b200/configio.py against files the reference program itself
writes with print_configs 1 (QMcBeaver/src/QMCConfigIO.cpp), byte for byte,
and the records' contents against the oracle at the recorded positions."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from qmcbeaver_b200.configio import ConfigIO, read_configs, record_dtype
from qmcbeaver_b200.system import make_system


def _random_records(N, k, seed=0):
    rng = np.random.default_rng(seed)
    r = np.zeros(k, record_dtype(N))
    r["n"] = N
    r["R"] = rng.standard_normal((k, N, 3))
    r["D1"] = rng.standard_normal(k) * 100
    r["D2"] = rng.standard_normal((k, N, 3))
    r["lnJ"] = rng.standard_normal(k)
    r["PE"] = -rng.random(k) * 50
    r["weight"] = rng.random(k)
    return r


@pytest.mark.parametrize("binary", [True, False])
def test_round_trip(tmp_path, binary):
    N = 7
    recs = _random_records(N, 9)
    path = str(tmp_path / "a.cfgs")
    io_ = ConfigIO(N, binary)
    io_.open(path, True)
    io_.write_records(recs[:5])
    for r in recs[5:]:
        io_.write(r["R"], r["D1"], r["D2"], r["lnJ"], r["PE"], r["weight"])
    io_.close()
    back = read_configs(path, N, binary)
    assert len(back) == 9
    for k in ("R", "D1", "D2", "lnJ", "PE", "weight"):
        if binary:
            assert np.array_equal(back[k], recs[k])
        else:  # fixed notation with 10 decimals (QMCConfigIO::setPrecision)
            assert np.allclose(back[k], recs[k], rtol=0, atol=6e-11)
    if binary:
        # 4-byte count + (6N + 4) doubles per record, no padding
        assert os.path.getsize(path) == 9 * (4 + 8 * (6 * N + 4))


def test_reader_rejects_wrong_electron_count(tmp_path):
    path = str(tmp_path / "b.cfgs")
    io_ = ConfigIO(4)
    io_.open(path, True)
    io_.write_records(_random_records(4, 2))
    io_.close()
    with pytest.raises(IOError):
        read_configs(path, 5)


def _reference_cfgs(workdir, system, steps, walkers, freq, seed):
    from oracle.refrun import REF_EXE
    flags = {"run_type": "variational", "sampling_method": "importance_sampling",
             "QF_modification_type": "umrigar93_unequalelectrons", "dt": 0.02, "number_of_walkers": walkers,
             "max_time_steps": steps, "equilibration_steps": 1, "one_e_per_iter": 1, "output_interval": 10 ** 6,
             "walkers_per_pass": 1, "print_configs": 1, "print_config_frequency": freq, "iseed": seed}
    system.to_ckmf(os.path.join(workdir, "run.ckmf"), flags)
    r = subprocess.run([REF_EXE, "run.ckmf"], cwd=workdir, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return os.path.join(workdir, "run.0.cfgs")


def test_reference_written_file(tmp_path):
    from oracle import refrun
    from oracle.evaluators import OracleEvaluator
    if not refrun.available():
        pytest.skip("reference build not present")
    s = make_system("dmc_6nuc_30e", seed=1)
    N = s.n_electrons
    path = _reference_cfgs(str(tmp_path), s, steps=90, walkers=4, freq=15, seed=-31)
    recs = read_configs(path, N)
    assert len(recs) >= 8 and len(recs) % 2 == 0
    # the file re-written by this writer is the reference's, byte for byte
    out = str(tmp_path / "again.cfgs")
    io_ = ConfigIO(N)
    io_.open(out, True)
    io_.write_records(recs)
    io_.close()
    assert open(out, "rb").read() == open(path, "rb").read()
    # pairs: the trial configuration with weight p, then the original with 1 - p,
    # differing in one electron
    t, o = recs[0::2], recs[1::2]
    assert np.allclose(t["weight"] + o["weight"], 1.0, rtol=0, atol=1e-12)
    assert all(np.count_nonzero(np.any(a != b, axis=1)) <= 1 for a, b in zip(t["R"], o["R"]))
    # the contents are the wavefunction's Slater part, ln J and PE at R
    orc = OracleEvaluator(s, qf_mod=2, dt=0.02)
    ws = orc.new_walkers(len(recs))
    orc.evaluate(ws, np.ascontiguousarray(recs["R"]), -1)
    res = orc.results(ws)
    ok = res["singular"] == 0
    rel = lambda a, b: np.abs(a - b) / np.maximum(np.abs(b), 1.0)
    assert np.max(rel(recs["D1"][ok], res["D_xx"][ok])) < 1e-9
    assert np.max(rel(recs["D2"][ok], orc.slater_grad(ws)[ok])) < 1e-9
    assert np.max(rel(recs["PE"][ok], res["potential"][ok])) < 1e-10
    # ln J of trial records; the reference's original-walker records carry a
    # stale ln J (QMCWalkerData::partialCopy does not copy U,
    # QMcBeaver/src/QMCWalkerData.cpp:32-54)
    okt = ok[0::2]
    assert np.max(rel(t["lnJ"][okt], res["U"][0::2][okt])) < 1e-10
