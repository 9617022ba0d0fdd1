"""The allocation-free branching entry point against the handle's branching.

qmcb_branch_weights_noalloc serves drivers that cannot allocate device
memory when they branch (a process whose HBM is all handed to its own pool,
or a step sequence that must not hit the device-wide synchronisation of
cudaMalloc / cudaFree).  Its scratch is a static device array shared by all
calls, so this test makes two calls in a row to check that the second call
does not see the first call's leftovers.  It sits in a file pytest collects
last, and passes both alone in a fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from qmcbeaver_b200.api import QMCB200Functions, load_library
from qmcbeaver_b200.desc import QMCB_DMC, run_params
from qmcbeaver_b200.system import make_system

pytestmark = pytest.mark.gpu


def test_noalloc_branching_matches_handle_branching():
    import torch
    torch.cuda.set_device(0)
    lib = load_library()
    s = make_system("vmc_water_10e", seed=1)
    W, seed = 3000, 4242
    f = QMCB200Functions(s, 2 * W, run_params(run_type=QMCB_DMC, seed=seed, limit_branching=0))
    R = s.initial_positions(W, seed=1)
    rng = np.random.default_rng(17)
    for step in (11, 12):  # two calls in a row share the static scratch
        w = np.exp(rng.normal(0.0, 1.3, W))
        w[rng.random(W) < 0.05] = 0.004
        # existing entry point: handle state, live list, device copies
        f.init_walkers(R)
        f.set_walker_weights(w)
        n_ref = f.branch(step)
        ref = f.get_walkers()["weight"]
        # allocation-free entry point: caller-owned device buffers
        d_in = torch.tensor(w, dtype=torch.float64, device="cuda")
        d_out = torch.full((2 * W,), -7.0, dtype=torch.float64, device="cuda")
        d_par = torch.full((2 * W,), -7, dtype=torch.int32, device="cuda")
        d_n = torch.zeros(1, dtype=torch.int32, device="cuda")
        rc = lib.qmcb_branch_weights_noalloc(C.c_void_p(d_in.data_ptr()), W, 2.0, 0.45, seed, step,
                                             C.c_void_p(d_out.data_ptr()), C.c_void_p(d_par.data_ptr()),
                                             C.c_void_p(d_n.data_ptr()), None)
        assert rc == 0, lib.qmcb_last_error(None)
        torch.cuda.synchronize()
        n = int(d_n.item())
        assert n == n_ref
        got = d_out[:n].cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=0, atol=0)
        par = d_par[:n].cpu().numpy()
        assert par.min() >= 0 and par.max() < W
        # survivors keep list order; every entry's weight comes from its source
        k = int(np.sum(par[1:] > par[:-1])) + 1
        assert k >= n - int(np.sum(w > 2.0))
    f.close()


def test_noalloc_rejects_oversize():
    lib = load_library()
    rc = lib.qmcb_branch_weights_noalloc(None, 70000, 2.0, 0.45, 1, 0, None, None, C.c_void_p(8), None)
    assert rc == 1 or rc == 5
    rc = lib.qmcb_branch_weights_noalloc(C.c_void_p(8), 65537, 2.0, 0.45, 1, 0, C.c_void_p(8), C.c_void_p(8),
                                         C.c_void_p(8), None)
    assert rc == 5
    assert b"QMCB_NOALLOC_MAX_WALKERS" in lib.qmcb_last_error(None)
