"""The reference's own test programs, unchanged, on the drop-in shim.

oracle/Makefile (`make shim`) compiles the reference's
TestNonPeriodic2D_MPI.cpp and TestNonPeriodic3D_MPI.cpp twice: against
mpi_b200/shim/NonPeriodic{2,3}D_B200.cpp over libhelm_b200.so (the GPU) and
against the reference's own CPU solver.  Both programs run here from the same
source: the shim's printed "Error = " (the device max-reduction of
ComputeError) must meet the reference's own bound, and the Tecplot files that
WriteFile leaves in Output/ must agree value for value.
"""
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


def _run(prog, cwd):
    os.makedirs(os.path.join(cwd, "Output"), exist_ok=True)
    r = subprocess.run([prog], cwd=cwd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    m = re.search(r"Error = (\S+)", r.stdout)
    assert m, r.stdout
    with open(os.path.join(cwd, "Output", "Solution-0000.tec")) as fh:
        head = [next(fh) for _ in range(3)]
        data = np.loadtxt(fh)
    return float(m.group(1)), head, data


@pytest.mark.parametrize("dim", [2, 3])
def test_reference_test_program_on_the_shim(cuda, tmp_path, dim):
    shim, ref = os.path.join(BIN, f"shim_test{dim}d"), os.path.join(BIN, f"ref_test{dim}d")
    if not (os.path.exists(shim) and os.path.exists(ref)):
        pytest.skip("the shim test programs are built only where the reference tree was present")
    err_gpu, head_gpu, tec_gpu = _run(shim, str(tmp_path / "gpu"))
    err_ref, head_ref, tec_ref = _run(ref, str(tmp_path / "ref"))
    # the stock manufactured solutions: 2D 512 x 512, N = 10 (52 elements,
    # Robin left end), 3D 64 x 32 x 250, N = 10 (25 elements); the reference
    # reaches ~1.7e-13 / 1.1e-13
    assert err_gpu < 1e-12 and err_ref < 1e-12, (err_gpu, err_ref)
    assert head_gpu == head_ref
    assert tec_gpu.shape == tec_ref.shape
    ncoord = dim
    assert np.abs(tec_gpu[:, :ncoord] - tec_ref[:, :ncoord]).max() < 2e-8  # printed with 8 decimals
    # U (the solution) and Exact columns agree to the printed precision
    assert np.abs(tec_gpu[:, ncoord:] - tec_ref[:, ncoord:]).max() < 2e-8
