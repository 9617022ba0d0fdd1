"""Synthetic molecule generator and the .ckmf writer."""
import math

import numpy as np
import pytest

from qmcbeaver_b200.system import (BasisFunction, WORKLOADS, make_system, system_from_arrays, system_to_arrays,
                                   _self_overlap)


@pytest.mark.parametrize("wl,ne,nn,nb", [("vmc_water_10e", 10, 3, 24), ("dmc_6nuc_30e", 30, 6, 120),
                                          ("mixed_20nuc_100e", 100, 20, 400)])
def test_workload_sizes(wl, ne, nn, nb):
    s = make_system(wl)
    assert (s.n_electrons, s.n_nuclei, s.n_basis) == (ne, nn, nb)
    assert s.n_alpha == s.n_beta == ne // 2
    assert s.mo.shape == (ne // 2, nb)


def test_water_geometry_and_basis_split():
    s = make_system("vmc_water_10e")
    assert list(s.Z) == [8, 1, 1]
    np.testing.assert_allclose(s.coords[1], [1.43, 1.11, 0.0])
    assert [len(fs) for fs in s.basis] == [14, 5, 5]


def test_contractions_normalised():
    s = make_system("dmc_6nuc_30e")
    for fs in s.basis:
        for f in fs:
            tot = sum(f.coefficients[i] * f.coefficients[j] * _self_overlap(f.powers, f.exponents[i], f.exponents[j])
                      for i in range(len(f.exponents)) for j in range(len(f.exponents)))
            assert abs(tot - 1.0) < 1e-12


def test_exponent_cache_guard():
    # the reference reuses exp(-a r^2) across an atom boundary when exponents
    # coincide (QMcBeaver/src/QMCBasisFunction.cpp:310,372-379)
    s = make_system("vmc_water_10e")
    s.basis[1][0] = BasisFunction("s", np.array([s.basis[0][-1].exponents[-1]]), np.array([1.0]))
    with pytest.raises(ValueError, match="stale exp cache"):
        s.check_exponent_cache()
    for wl in WORKLOADS:
        make_system(wl).check_exponent_cache()


def test_round_trip_arrays():
    s = make_system("dmc_6nuc_30e")
    t = system_from_arrays(system_to_arrays(s))
    assert t.labels == s.labels and t.n_basis == s.n_basis
    np.testing.assert_array_equal(t.mo, s.mo)
    assert t.en_up["H"].num == s.en_up["H"].num if "H" in s.en_up else True


def test_ckmf_writer_sections(tmp_path):
    s = make_system("vmc_water_10e")
    p = tmp_path / "w.ckmf"
    s.to_ckmf(str(p))
    txt = p.read_text()
    for sec in ("&flags", "&geometry", "&basis", "&wavefunction", "&Jastrow", "Alpha Occupation", "FixedCuspPade"):
        assert sec in txt
    assert "one_e_per_iter\n 1" in txt and "use_three_body_jastrow\n 0" in txt


def test_pade_fixed_cusp_values():
    from qmcbeaver_b200.system import Pade
    p = Pade.fixed_cusp(0.5, 1.0)
    u, du, d2u = p.evaluate(2.0)
    assert math.isclose(u, 0.5 * 2 / 3)
    assert math.isclose(du, 0.5 / 9)
    assert math.isclose(d2u, -2 * 0.5 / 27)
