"""Snapshot files in the reference's format (Output::WriteSolutionSnapshot,
Output.cpp:145-330): VTK rectilinear grids with the reference's field names
at the cell centres; the arrays read back equal the interior state."""
import numpy as np

from m2c_b200 import abi, cases, output


def test_vtr_round_trip(tmp_path):
    g, s, mats, ls, V, ID, PHI = cases.bubble_case(12, nbubbles=1, mesh=cases.stretch)
    path = str(tmp_path / output.frame_name("solution", 7))
    assert path.endswith("solution_0007.vtr")
    output.write_vtr(path, g, V, ID, PHI)
    d = output.read_vtr(path)
    inner = np.s_[1:-1, 1:-1, 1:-1]
    assert np.array_equal(d["density"], V[inner][..., 0].ravel())
    assert np.array_equal(d["velocity"], V[inner][..., 1:4].reshape(-1, 3))
    assert np.array_equal(d["pressure"], V[inner][..., 4].ravel())
    assert np.array_equal(d["materialid"], ID[inner].ravel())
    assert np.array_equal(d["levelset0"], PHI[inner].ravel())
    xc, yc, zc = abi.cell_centres(g)
    assert np.array_equal(d["x"], xc) and np.array_equal(d["y"], yc) and np.array_equal(d["z"], zc)
    head = open(path, "rb").read(400).decode(errors="ignore")
    assert 'type="RectilinearGrid"' in head and 'WholeExtent="0 11 0 11 0 11"' in head
