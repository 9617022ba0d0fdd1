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


def _noalloc(lib, w, thr, fuse, seed, step):
    import torch
    n_in = len(w)
    d_in = torch.tensor(w, dtype=torch.float64, device="cuda")
    d_out = torch.full((2 * n_in,), -7.0, dtype=torch.float64, device="cuda")
    d_par = torch.full((2 * n_in,), -7, dtype=torch.int32, device="cuda")
    d_n = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.qmcb_branch_weights_noalloc(C.c_void_p(d_in.data_ptr()), n_in, thr, fuse, seed, step,
                                         C.c_void_p(d_out.data_ptr()), C.c_void_p(d_par.data_ptr()),
                                         C.c_void_p(d_n.data_ptr()), None)
    assert rc == 0, lib.qmcb_last_error(None)
    torch.cuda.synchronize()
    n = int(d_n.item())
    return d_out[:n].cpu().numpy(), d_par[:n].cpu().numpy()


def test_noalloc_branching_matches_handle_branching():
    import torch
    torch.cuda.set_device(0)
    lib = load_library()
    s = make_system("vmc_water_10e", seed=1)
    W, seed = 3000, 4242
    R = s.initial_positions(W, seed=1)
    rng = np.random.default_rng(17)
    for fuse in (0.45, 1.5):  # 1.5: fused pairs can exceed the branching threshold
        f = QMCB200Functions(s, 3 * W, run_params(run_type=QMCB_DMC, seed=seed, limit_branching=0,
                                                  fusion_threshold=fuse))
        f.init_walkers(R)
        n_live = W
        # two calls in a row share the static scratch; the second runs on the
        # handle's reordered live list (deaths removed, copies appended), so
        # the fusion draws must follow the list position, not the slot
        for step in (11, 12):
            w = np.exp(rng.normal(0.0, 1.3, n_live))
            w[rng.random(n_live) < 0.05] = 0.004
            # existing entry point: handle state, live list, device copies
            f.set_walker_weights(w)
            n_ref = f.branch(step)
            ref = f.get_walkers()["weight"]
            # allocation-free entry point: caller-owned device buffers
            got, par = _noalloc(lib, w, 2.0, fuse, seed, step)
            assert len(got) == n_ref
            np.testing.assert_allclose(got, ref, rtol=0, atol=0)
            assert par.min() >= 0 and par.max() < n_live
            # survivors keep list order, split copies follow with their sources in order
            assert np.count_nonzero(np.diff(par) <= 0) <= 1
            n_live = n_ref
        f.close()


def test_noalloc_rejects_oversize():
    import torch
    torch.cuda.set_device(0)
    lib = load_library()
    n_big = 65537
    d_in = torch.ones(n_big, dtype=torch.float64, device="cuda")
    d_out = torch.full((2 * n_big,), -7.0, dtype=torch.float64, device="cuda")
    d_par = torch.full((2 * n_big,), -7, dtype=torch.int32, device="cuda")
    d_n = torch.full((1,), -3, dtype=torch.int32, device="cuda")
    args = (C.c_void_p(d_out.data_ptr()), C.c_void_p(d_par.data_ptr()), C.c_void_p(d_n.data_ptr()), None)
    rc = lib.qmcb_branch_weights_noalloc(C.c_void_p(d_in.data_ptr()), n_big, 2.0, 0.45, 1, 0, *args)
    assert rc == 5
    assert b"QMCB_NOALLOC_MAX_WALKERS" in lib.qmcb_last_error(None)
    torch.cuda.synchronize()
    assert int(d_n.item()) == -3 and float(d_out.min()) == -7.0  # nothing was launched
    # the limit itself is accepted
    rc = lib.qmcb_branch_weights_noalloc(C.c_void_p(d_in.data_ptr()), 65536, 2.0, 0.45, 1, 0, *args)
    assert rc == 0, lib.qmcb_last_error(None)
    torch.cuda.synchronize()
    assert int(d_n.item()) == 65536
