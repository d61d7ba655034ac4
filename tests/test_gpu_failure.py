"""Failure handling with host-made failures (no GPU fault): a device
allocation that fails during set-up, the construct kernel's bounded staging
wait running out, and set-up arguments the reference's solver would have to
handle (ants = 0, fewer customers than candidates)."""
import numpy as np
import pytest

from vehicleroutingproblem_b200 import _native as N
from vehicleroutingproblem_b200 import instances as I

pytestmark = pytest.mark.gpu


def _fresh(inst, epochs, **kw):
    with N.Context(0) as c:
        c.setup_instance(inst, **kw)
        st = c.run(epochs)
        return st.global_best, c.tau()


@pytest.mark.parametrize("at", [1, 7, 16, 28])
def test_allocation_failure_during_setup(at):
    import torch
    inst = I.uniform_instance(150, 3, 931)
    kw = dict(ants=32, cand_k=16, seed=4)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    with N.Context(0) as c:
        c.debug_inject(1, at)
        with pytest.raises(N.AcoError) as err:
            c.setup_instance(inst, **kw)
        assert err.value.status == N.ACO_ERR_ALLOCATION
        # nothing of the failed set-up stays allocated
        assert abs(torch.cuda.mem_get_info()[0] - free0) < (8 << 20)
        with pytest.raises(N.AcoError):
            c.run(1)  # no usable set-up
        c.setup_instance(inst, **kw)  # the injection fired once
        st = c.run(10)
        gb, tau = _fresh(inst, 10, **kw)
        assert st.global_best == gb and np.array_equal(c.tau(), tau)


def test_staging_wait_timeout_reports_and_recovers():
    inst = I.uniform_instance(300, 5, 932)
    kw = dict(ants=64, cand_k=24, seed=6)
    with N.Context(0) as c:
        c.setup_instance(inst, **kw)
        c.debug_inject(2, 1)
        with pytest.raises(N.AcoError) as err:
            c.run(3)
        assert err.value.status == N.ACO_ERR_BACKEND
        assert c.state().error & 1
        c.setup_instance(inst, **kw)  # a set-up clears the injection and the state
        st = c.run(12)
        assert st.error == 0 and st.epochs == 12
        gb, tau = _fresh(inst, 12, **kw)
        assert st.global_best == gb and np.array_equal(c.tau(), tau)


def test_setup_defaults_and_clamps():
    inst = I.uniform_instance(20, 2, 933)
    with N.Context(0) as c:
        c.setup_instance(inst, ants=0, cand_k=32, seed=1)
        assert (c.n, c.m, c.k) == (20, 256, 20)  # m = 0 -> 256; k clamped to n
        st = c.run(5)
        assert st.epochs == 5 and np.isfinite(st.global_best)
