"""The output writers against the reference's own WriteFile (GPU: a plan needs a device).

tests/golden/writer_2d.tec / writer_3d.tec are the files the reference's
WriteFile (TECPLOT branch, NonPeriodic2D_MPI.cpp:571-598,
NonPeriodic3D_MPI.cpp:713-741) wrote for the fields in writer_fields.npz
(tests/golden/make_golden.py); helm_write_tecplot must reproduce them byte for
byte.  The VTK writer (the reference's VISIT branch, compiled out of its build)
is checked for structure and values.
"""
import math

import numpy as np
import pytest
import torch

from mpi_b200 import NonPeriodic2D, NonPeriodic3D, Periodic2D
from tests.helpers import GOLDEN, golden

pytestmark = pytest.mark.gpu


def _read(name):
    with open(f"{GOLDEN}/{name}") as fh:
        return fh.read()


def test_tecplot_matches_reference_2d(cuda, tmp_path):
    g = golden("writer_fields")
    xl, xr, yl, yr = [float(v) for v in g["dom2"]]
    p = NonPeriodic2D(8, 10, 5, xl, xr, yl, yr, Lambda=1.0)
    path = str(tmp_path / "sol.tec")
    p.WriteFile(torch.from_numpy(g["u2"]), path, exact=lambda x, y, z: math.sin(x) * math.cos(y))
    assert open(path).read() == _read("writer_2d.tec")


def test_tecplot_matches_reference_3d(cuda, tmp_path):
    g = golden("writer_fields")
    xl, xr, yl, yr, zl, zr = [float(v) for v in g["dom3"]]
    p = NonPeriodic3D(4, 4, 8, 4, xl, xr, yl, yr, zl, zr, Lambda=1.0)
    path = str(tmp_path / "sol.tec")
    p.WriteFile(torch.from_numpy(g["u3"]).cuda(), path, exact=lambda x, y, z: math.sin(x) * math.cos(y) * z)
    assert open(path).read() == _read("writer_3d.tec")


def test_vtk_structure_and_values(cuda, tmp_path):
    g = golden("writer_fields")
    u = g["u2"]
    p = Periodic2D(8, 10, 5, 0.5, 2.0, -1.0, 1.0, Lambda=1.0)
    path = str(tmp_path / "sol.vtk")
    p.WriteFile(torch.from_numpy(u), path, fmt="vtk")
    lines = open(path).read().splitlines()
    assert lines[:4] == ["# vtk DataFile Version 3.1", "Helmholtz solver", "ASCII", "DATASET STRUCTURED_GRID"]
    assert lines[4] == "DIMENSIONS 8 10 1" and lines[5] == "POINTS 80 FLOAT"
    pts = np.array([[float(t) for t in l.split("\t")] for l in lines[6:86]])
    nodes = p.grid()[0].numpy()
    assert np.allclose(pts[:8, 0], 0.5 + np.arange(8) * 1.5 / 8, atol=1e-8)
    assert np.allclose(pts[::8, 1], np.concatenate([nodes[0:5], nodes[4:9]]), atol=1e-8)
    assert lines[87] == "POINT_DATA 80" and lines[88] == "SCALARS Phi float"
    vals = np.array([float(l) for l in lines[90:170]])
    # points run element, GLL node, x (x fastest)
    assert np.allclose(vals, u.transpose(0, 2, 1).ravel(), atol=5e-9)
