"""Out-of-memory paths of plan creation, by host-side fault injection
(helm_debug_fail_alloc): each device allocation of a plan is made to fail in
turn; creation must return HELM_ERR_OOM with its message, free everything it
had allocated, and leave the library usable (the next creation succeeds and
solves correctly).  No GPU fault is involved: the failing call is the
library's own allocation wrapper."""
import numpy as np
import pytest
import torch

from mpi_b200 import BatchNonPeriodic2D, Helmholtz3DFD, NonPeriodic3D
from mpi_b200 import _lib as L
from mpi_b200._lib import HelmError
from oracle import oracle as O
from tests.helpers import max_rel

pytestmark = pytest.mark.gpu


def _free_bytes():
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def _inject_each(make, max_allocs=200):
    """Fail allocation n = 0, 1, ... of `make` until it succeeds; every failure
    is HELM_ERR_OOM and leaks no device memory.  Returns the number of failing
    allocations tried and the successful object."""
    lib = L.lib()
    make().close()  # warm caches (autotune results, module load) outside the count
    base = _free_bytes()
    for n in range(max_allocs):
        lib.helm_debug_fail_alloc(n)
        try:
            obj = make()
        except HelmError as e:
            assert e.status == L.HELM_ERR_OOM, e
            assert "injected" in lib.helm_last_error().decode()
            lost = base - _free_bytes()
            assert lost < (4 << 20), f"allocation {n}: {lost} bytes not returned"
            continue
        finally:
            lib.helm_debug_fail_alloc(-1)
        return n, obj
    raise AssertionError("creation kept failing")


class _Closing:
    def __init__(self, obj, close):
        self.obj, self._close = obj, close

    def close(self):
        self._close()


def test_plan_create_oom_3d(cuda):
    def make():
        p = NonPeriodic3D(32, 16, 17, 17, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=2.0)
        return _Closing(p, p.DestroyPDEPlan)

    n, made = _inject_each(make)
    assert n >= 5  # the spectrum, twiddles, per-shift data, transforms ...
    p = made.obj
    rng = np.random.default_rng(1)
    f = rng.standard_normal((32, 16, 17))
    z = np.zeros((32, 16))
    ref = O.solve3d(f, z, z, Lx=1.0, Ly=2.0, Lz=1.5, lam=2.0)
    u = p.SolvePDE(torch.from_numpy(f).cuda()).cpu().numpy()
    assert max_rel(u, ref) < 1e-12
    p.DestroyPDEPlan()


def test_plan_create_oom_fd_and_batch(cuda):
    def make_fd():
        p = Helmholtz3DFD(16, 8, 600, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0)
        return _Closing(p, p.DestroyPDEPlan)

    n, made = _inject_each(make_fd)
    assert n >= 3
    made.close()

    def make_batch():
        b = BatchNonPeriodic2D([16, 32, 16], [9, 17, 9], [1.0, 2.0, 3.0], 0.0, 1.0, -1.0, 1.0)
        return _Closing(b, b.destroy)

    n, made = _inject_each(make_batch)
    assert n >= 2
    made.close()


def test_fault_hook_disarms(cuda):
    lib = L.lib()
    lib.helm_debug_fail_alloc(0)
    with pytest.raises(HelmError):
        NonPeriodic3D(16, 8, 9, 9, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0)
    # fired once, disarmed: the next creation succeeds
    p = NonPeriodic3D(16, 8, 9, 9, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0)
    p.DestroyPDEPlan()
