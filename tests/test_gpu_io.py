"""PencilDcmp::IO (src/pencilDcmp.cpp:1827-1832 -> Phdf5::writeMultiBlockCellCenter,
src/phdf5.cpp:1299-1808) through the C ABI: soln/Pxdmf3d<app>.xmf, the
reference's file name and grid structure (a Collection "AMR" of one Uniform
grid "mesh0", the cell-centred attribute "Q" = the real part of P), with the
values in a raw float64 file referenced as an XDMF Binary item (no HDF5)."""
import xml.etree.ElementTree as ET

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_io_writes_the_solution_for_paraview(tmp_path, monkeypatch):
    import pittpack_b200 as pp

    monkeypatch.chdir(tmp_path)
    nx, ny, nz = 12, 10, 8
    box = [0.0, 2.0, -1.0, 1.0, 0.5, 1.5]
    f = np.random.default_rng(4).standard_normal((nz, ny, nx))
    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary("PPNNDD")
        M.setBox(box)
        M.assignRhsComplex(f + 1j * f[::-1])
        with pytest.raises(pp.PittPackError) as e:
            M.IO(3, 2, 0)  # before a solve
        assert e.value.code == 25
        M.pittPack()
        P = M.getSolution()
        M.IO(3, 2, 0)
        with pytest.raises(pp.PittPackError) as e:
            M.IO(3, 5, 0)  # dir outside 0..2
        assert e.value.code == 19
    root = ET.parse(tmp_path / "soln" / "Pxdmf3d3.xmf").getroot()
    coll = root.find("Domain/Grid")
    assert coll.get("Name") == "AMR" and coll.get("GridType") == "Collection"
    grid = coll.find("Grid")
    assert grid.get("Name") == "mesh0" and grid.get("GridType") == "Uniform"
    topo = grid.find("Topology")
    assert topo.get("TopologyType") == "3DCoRectMesh"
    assert [int(v) for v in topo.get("Dimensions").split()] == [nz + 1, ny + 1, nx + 1]
    origin, spacing = grid.findall("Geometry/DataItem")
    assert np.allclose([float(v) for v in origin.text.split()], [box[4], box[2], box[0]], rtol=0, atol=0)
    assert np.allclose([float(v) for v in spacing.text.split()],
                       [(box[5] - box[4]) / nz, (box[3] - box[2]) / ny, (box[1] - box[0]) / nx], rtol=1e-16)
    attr = grid.find("Attribute")
    assert attr.get("Name") == "Q" and attr.get("Center") == "Cell"
    item = attr.find("DataItem")
    assert item.get("Format") == "Binary" and item.get("Endian") == "Little" and item.get("Precision") == "8"
    assert [int(v) for v in item.get("Dimensions").split()] == [nz, ny, nx]
    Q = np.fromfile(tmp_path / "soln" / item.text.strip(), dtype="<f8").reshape(nz, ny, nx)
    assert np.array_equal(Q, P.real)
