"""Bounded device waits that run out, without faulting or hanging the GPU.

The colouring's grid barriers and the seed network's tensor-core mbarrier
waits give up after a limit, set IGR_ERR_TIMEOUT and return.  Here the test
hooks make the wait run out by construction: the grid barrier waits for one
arrival that never comes, and the GEMM first waits on an mbarrier phase that
nothing completes (before it issues any MMA).  Each call must return the
timeout status, and the next call with the hooks reset must give the oracle's
result on the same context.
"""
import numpy as np
import pytest

import instantgr_b200 as ig
import cases
from oracle_py import color as orc_color, seed_grad

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _reset_hooks():
    ig.set_test_hook(ig.HOOK_RESET)
    yield
    ig.set_test_hook(ig.HOOK_RESET)


def test_colouring_barrier_wait_runs_out_and_context_stays_usable():
    X, Y = 64, 48
    args = cases.color_case(31, X, Y, 300)
    g = cases.grid_case(1, X=X, Y=Y)
    c = ig.Ctx(g["L"], g["X"], g["Y"], g["DIR"], g["xlen"], g["ylen"], g["unit_wire"], g["unit_via"], g["short"],
               g["cap"])
    ig.set_test_hook(ig.HOOK_WAIT_NS, 1_000_000)  # 1 ms
    ig.set_test_hook(ig.HOOK_BARRIER_PHANTOM, 1)
    with pytest.raises(ig.IgrError) as e:
        c.color_batches(*args, sparsity=3)
    assert e.value.code == -6  # IGR_ERR_TIMEOUT
    ig.set_test_hook(ig.HOOK_RESET)
    b_gpu, nb_gpu = c.color_batches(*args, sparsity=3)
    b_orc, nb_orc = orc_color(X, Y, *args, sparsity=3)
    assert nb_gpu == nb_orc and np.array_equal(b_gpu, b_orc)
    c.close()


def test_seed_gemm_mbarrier_wait_runs_out_and_model_stays_usable():
    m = ig.Seed(3)
    m.set_tile(32, 4)
    p = m.params()
    rng = np.random.default_rng(5)
    x = rng.normal(0, 1, (1, 32, 32, 16)).astype(np.float32)
    t = np.abs(rng.normal(0, 1, (1, 32, 32, 16))).astype(np.float32)
    ig.set_test_hook(ig.HOOK_WAIT_NS, 1_000_000)
    ig.set_test_hook(ig.HOOK_MBAR_PROBE, 1)
    with pytest.raises(ig.IgrError) as e:
        m.grad(x, t)
    assert e.value.code == -6  # IGR_ERR_TIMEOUT
    ig.set_test_hook(ig.HOOK_RESET)
    loss_g, grad_g = m.grad(x, t)
    loss_o, grad_o = seed_grad(x, t, p, 4, rounded=True)
    assert abs(loss_g - loss_o) <= 1e-3 * loss_o
    assert np.linalg.norm(grad_g - grad_o) <= 3e-2 * np.linalg.norm(grad_o)
    m.close()
