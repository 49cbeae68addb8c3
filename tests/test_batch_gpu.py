"""Batched independent 2D solves of uneven sizes (helm2d_batch_*): every
problem against the oracle's own solve of it (oracle/helm_oracle.c:
orc_solve2d), against a single-problem plan, and against the manufactured exact
solution; graph replay against direct launches.  Tolerances: FP64 1e-12 max
relative, FP32 with refinement 1e-10 relative L2, FP32 1e-5."""
import math

import numpy as np
import pytest
import torch

from mpi_b200 import BatchNonPeriodic2D, NonPeriodic2D
from mpi_b200 import workloads as W
from oracle import oracle as O
from tests.helpers import max_rel, rel_l2

pytestmark = pytest.mark.gpu

TWO_PI = 2.0 * math.pi


def _small_batch(seed=3, n=14):
    rng = np.random.default_rng(seed)
    Nx = [int(v) for v in rng.choice((8, 16, 32, 64), n)]
    P = [int(v) for v in rng.choice((5, 9, 17, 33), n)]
    lam = [float(v) for v in 10.0 ** rng.uniform(-2, 4, n)]
    fs = [rng.standard_normal((a, b)) for a, b in zip(Nx, P)]
    return Nx, P, lam, fs


def _solve_batch(Nx, P, lam, fs, precision, graph=True):
    b = BatchNonPeriodic2D(Nx, P, lam, 0.0, TWO_PI, -1.0, 1.0, precision=precision)
    b.set_graph(graph)
    f = b.pack([torch.from_numpy(x) for x in fs]).cuda()
    u = b.solve(f)
    torch.cuda.synchronize()
    return b, [x.cpu().numpy() for x in b.unpack(u)]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32_refine", 1e-10), ("fp32", 1e-5)])
def test_batch_matches_oracle(cuda, precision, tol):
    Nx, P, lam, fs = _small_batch()
    b, us = _solve_batch(Nx, P, lam, fs, precision)
    assert b.info()["classes"] == len(set(zip(Nx, P)))
    for f, u, la in zip(fs, us, lam):
        ref = O.solve2d(f, np.zeros(f.shape[0]), np.zeros(f.shape[0]), Lx=TWO_PI, Ly=2.0, lam=la)
        err = max_rel(u, ref) if precision == "fp64" else rel_l2(u, ref)
        assert err < tol, (f.shape, la, err)


def test_batch_equals_single_plans(cuda):
    Nx, P, lam, fs = _small_batch(seed=5, n=9)
    _, us = _solve_batch(Nx, P, lam, fs, "fp64")
    for f, u, nx, p, la in zip(fs, us, Nx, P, lam):
        pl = NonPeriodic2D(nx, p, p, 0.0, TWO_PI, -1.0, 1.0, Lambda=la)
        v = pl.SolvePDE(torch.from_numpy(f).cuda()).cpu().numpy()
        assert max_rel(u, v) < 1e-13


def test_batch_graph_replay_and_recapture(cuda):
    Nx, P, lam, fs = _small_batch(seed=7, n=10)
    b = BatchNonPeriodic2D(Nx, P, lam, 0.0, TWO_PI, -1.0, 1.0, precision="fp32_refine")
    f = b.pack([torch.from_numpy(x) for x in fs]).cuda()
    b.set_graph(False)
    u_direct = b.solve(f).clone()
    b.set_graph(True)
    u1 = b.solve(f).clone()
    u2 = b.solve(f).clone()           # replay of the same graph
    f2 = (2.0 * f).contiguous()       # new pointers: captured again
    u3 = b.solve(f2).clone()
    torch.cuda.synchronize()
    assert torch.equal(u1, u_direct) and torch.equal(u2, u_direct)
    assert (u3 - 2.0 * u_direct).abs().max().item() <= 1e-12 * u_direct.abs().max().item()


def test_batch_on_side_stream(cuda):
    Nx, P, lam, fs = _small_batch(seed=11, n=6)
    b = BatchNonPeriodic2D(Nx, P, lam, 0.0, TWO_PI, -1.0, 1.0)
    f = b.pack([torch.from_numpy(x) for x in fs]).cuda()
    ref = b.solve(f).clone()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        u = b.solve(f, stream=s)
    s.synchronize()
    assert torch.equal(u, ref)


def test_batch_one_launch_and_fallback(cuda):
    """FP64 / refined batches in range run as one persistent kernel launch;
    FP32 batches and batches with a problem outside its range (Nx = 1024) run
    the size classes (three kernels each); both match single-problem plans."""
    Nx, P, lam, fs = _small_batch(seed=13, n=8)
    b, us = _solve_batch(Nx, P, lam, fs, "fp64")
    assert b.info()["kernels_per_solve"] == 1
    assert b.device_status() == 0
    b32, _ = _solve_batch(Nx, P, lam, fs, "fp32")
    assert b32.info()["kernels_per_solve"] == 3 * len(set(zip(Nx, P)))
    Nx2, P2, lam2 = Nx + [1024], P + [9], lam + [3.0]
    fs2 = fs + [np.random.default_rng(1).standard_normal((1024, 9))]
    b2, us2 = _solve_batch(Nx2, P2, lam2, fs2, "fp64")
    assert b2.info()["kernels_per_solve"] == 3 * len(set(zip(Nx2, P2)))
    for u, v in zip(us, us2):
        assert max_rel(u, v) < 1e-13
    pl = NonPeriodic2D(1024, 9, 9, 0.0, TWO_PI, -1.0, 1.0, Lambda=3.0)
    assert max_rel(us2[-1], pl.SolvePDE(torch.from_numpy(fs2[-1]).cuda()).cpu().numpy()) < 1e-13


def test_batch_full_size_512(cuda):
    """512 problems, Nx in {32..512}, GLL order in {16..128}, lambda log-uniform in
    [1e-2, 1e4], the manufactured 2D problem: FP32 + refinement against FP64 per
    problem, both against the exact solution, and a sample against the oracle."""
    Nx, P, lam, fs, us_exact = W.batch_2d(512, seed=1237)
    b64, u64 = _solve_batch(Nx, P, lam, fs, "fp64")
    b32r, u32r = _solve_batch(Nx, P, lam, fs, "fp32_refine")
    assert b64.info()["kernels_per_solve"] == 1 and b32r.info()["kernels_per_solve"] == 1
    assert b64.device_status() == 0 and b32r.device_status() == 0
    worst = max(rel_l2(a, b) for a, b in zip(u32r, u64))
    assert worst < 1e-10, worst
    assert max(rel_l2(a, e) for a, e in zip(u64, us_exact)) < 1e-11
    for i in range(0, 512, 37):
        f = fs[i]
        ref = O.solve2d(f, np.zeros(f.shape[0]), np.zeros(f.shape[0]), Lx=TWO_PI, Ly=2.0, lam=lam[i])
        assert rel_l2(u32r[i], ref) < 1e-10
        assert max_rel(u64[i], ref) < 1e-11
