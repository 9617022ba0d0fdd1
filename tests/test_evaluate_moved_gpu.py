"""The single-electron evaluate entry point (qmcb_evaluate_moved: only the
moved electron's position goes up, only the selected outputs come back)
against qmcb_evaluate, and the slot allocator of the evaluate entry points."""
import numpy as np
import pytest

from qmcbeaver_b200.api import (OUT_ALL, OUT_E_LOCAL, OUT_MOD_GRAD, OUT_PSI, OUT_STATUS, QMCB200Functions,
                                QMCBError)
from qmcbeaver_b200.desc import QMCB_PREC_FP64, QMCB_PREC_INT8_SLICES
from qmcbeaver_b200.system import make_system

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("wl,prec", [("dmc_6nuc_30e", QMCB_PREC_FP64), ("vmc_threebody_16e", QMCB_PREC_FP64),
                                     ("vmc_multidet_12e", QMCB_PREC_FP64), ("dmc_6nuc_30e", QMCB_PREC_INT8_SLICES)])
def test_moved_equals_full_positions(wl, prec):
    s = make_system(wl, seed=2)
    W = 300
    a = QMCB200Functions(s, W, qf_modification=2, dt=0.01, precision=prec)
    b = QMCB200Functions(s, W, qf_modification=2, dt=0.01, precision=prec)
    R = s.initial_positions(W, seed=3)
    sl = np.arange(W)
    a.evaluate(sl, R, -1)
    b.evaluate(sl, R, -1)
    rng = np.random.default_rng(1)
    for m in range(2 * s.n_electrons):
        e = m % s.n_electrons
        R[:, e] += 0.15 * rng.standard_normal((W, 3))
        x = a.evaluate(sl, R, e)
        y = b.evaluate_moved(sl, R[:, e], e)
        for k in ("log_abs_psi", "sign", "grad", "mod_grad", "lap", "e_local", "pe", "status"):
            np.testing.assert_array_equal(x[k], y[k], err_msg=f"{wl} move {m} {k}")
    a.close()
    b.close()


def test_moved_writes_only_selected_outputs():
    s = make_system("vmc_water_10e", seed=1)
    W = 64
    f = QMCB200Functions(s, W)
    R = s.initial_positions(W, seed=2)
    sl = np.arange(W)
    full = f.evaluate(sl, R, -1)
    R[:, 3] += 0.1
    mask = OUT_PSI | OUT_MOD_GRAD | OUT_E_LOCAL | OUT_STATUS
    out = dict(log_abs_psi=np.full(W, 7.0), sign=np.full(W, 7.0), grad=np.full((W, s.n_electrons, 3), 7.0),
               mod_grad=np.full((W, s.n_electrons, 3), 7.0), lap=np.full(W, 7.0), e_local=np.full(W, 7.0),
               pe=np.full((W, 3), 7.0), status=np.full(W, 7, np.uint8))
    f.evaluate_moved(sl, R[:, 3], 3, mask, out=out)
    assert np.all(out["grad"] == 7.0) and np.all(out["lap"] == 7.0) and np.all(out["pe"] == 7.0)
    assert not np.any(out["e_local"] == 7.0) and not np.any(out["mod_grad"] == 7.0)
    assert np.all(out["status"] <= 3)
    # an output selected in the mask without a buffer is refused before any launch
    sl32, r3 = sl.astype(np.int32), np.ascontiguousarray(R[:, 3])
    rc = f.lib.qmcb_evaluate_moved(f.h, 3, sl32.ctypes.data, W, r3.ctypes.data, OUT_ALL, *([None] * 8))
    assert rc == 1 and b"NULL" in f.lib.qmcb_last_error(f.h)
    f.close()
    assert np.isfinite(full["e_local"]).all()


def test_page_locked_inputs_equal_copied_inputs():
    """Slots and moved positions in page-locked host memory (copied by DMA
    straight from the caller's buffers): the same results as pageable inputs,
    call after call, with a permuted slot list."""
    import torch
    torch.cuda.set_device(0)
    s = make_system("dmc_6nuc_30e", seed=2)
    W, N = 150, s.n_electrons
    a = QMCB200Functions(s, W, qf_modification=2, dt=0.01)
    b = QMCB200Functions(s, W, qf_modification=2, dt=0.01)
    R = s.initial_positions(W, seed=3)
    sl = np.arange(W)[::-1].copy()  # a permuted slot list
    a.evaluate(sl, R, -1)
    b.evaluate(sl, R, -1)
    sl_pin = torch.tensor(sl, dtype=torch.int32).pin_memory().numpy()
    r_pin = torch.zeros((W, 3), dtype=torch.float64).pin_memory().numpy()
    rng = np.random.default_rng(6)
    for m in range(N + 2):
        e = m % N
        R[:, e] += 0.15 * rng.standard_normal((W, 3))
        r_pin[:] = R[:, e]
        x = a.evaluate_moved(sl, np.ascontiguousarray(R[:, e]), e)
        y = b.evaluate_moved(sl_pin, r_pin, e)
        for k in ("log_abs_psi", "sign", "mod_grad", "e_local", "pe", "status"):
            np.testing.assert_array_equal(x[k], y[k], err_msg=f"move {m} {k}")
    a.close()
    b.close()


@pytest.mark.parametrize("entry", ["moved", "all_positions"])
def test_page_locked_outputs_equal_copied_outputs(entry):
    """Outputs in mapped page-locked host memory are stored by the kernel
    over the bus; they must equal the outputs copied back into pageable
    arrays, and outputs not selected stay untouched."""
    import torch
    torch.cuda.set_device(0)
    s = make_system("dmc_6nuc_30e", seed=2)
    W, N = 200, s.n_electrons
    a = QMCB200Functions(s, W, qf_modification=2, dt=0.01)
    b = QMCB200Functions(s, W, qf_modification=2, dt=0.01)
    R = s.initial_positions(W, seed=3)
    sl = np.arange(W)
    a.evaluate(sl, R, -1)
    b.evaluate(sl, R, -1)
    shapes = (("log_abs_psi", (W,), torch.float64), ("sign", (W,), torch.float64),
              ("grad", (W, N, 3), torch.float64), ("mod_grad", (W, N, 3), torch.float64),
              ("lap", (W,), torch.float64), ("e_local", (W,), torch.float64), ("pe", (W, 3), torch.float64),
              ("status", (W,), torch.uint8))
    pin = {k: torch.full(shp, 7, dtype=dt).pin_memory().numpy() for k, shp, dt in shapes}
    mask = OUT_PSI | OUT_MOD_GRAD | OUT_E_LOCAL | OUT_STATUS
    rng = np.random.default_rng(4)
    for m in range(N + 3):
        e = m % N
        R[:, e] += 0.15 * rng.standard_normal((W, 3))
        if entry == "moved":
            x = a.evaluate_moved(sl, R[:, e], e, mask)
            y = b.evaluate_moved(sl, R[:, e], e, mask, out=pin)
            keys = ("log_abs_psi", "sign", "mod_grad", "e_local", "status")
            for k in ("grad", "lap", "pe"):
                assert np.all(pin[k] == 7), (m, k)
        else:
            x = a.evaluate(sl, R, e)
            rc = b.lib.qmcb_evaluate(b.h, e, np.ascontiguousarray(sl, dtype=np.int32).ctypes.data, W,
                                     np.ascontiguousarray(R).ctypes.data,
                                     *[pin[k].ctypes.data for k, _, _ in shapes])
            assert rc == 0, b.lib.qmcb_last_error(b.h)
            y = pin
            keys = [k for k, _, _ in shapes]
        for k in keys:
            np.testing.assert_array_equal(x[k], y[k], err_msg=f"{entry} move {m} {k}")
    a.close()
    b.close()


def test_slot_allocator():
    s = make_system("vmc_water_10e", seed=1)
    f = QMCB200Functions(s, 5)
    got = [f.alloc_slot() for _ in range(5)]
    assert sorted(got) == [0, 1, 2, 3, 4]
    with pytest.raises(QMCBError, match="in use"):
        f.alloc_slot()
    f.free_slot(got[2])
    assert f.alloc_slot() == got[2]
    f.free_slot(got[0])
    with pytest.raises(QMCBError, match="not handed out"):
        f.free_slot(got[0])
    with pytest.raises(QMCBError, match="not handed out"):
        f.free_slot(99)
    f.close()
