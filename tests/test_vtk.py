"""Legacy ASCII VTK writer and the cell→node stress projection (host code), checked
against the expectations of the reference's test/test_vtk.jl and
test/test_postprocess_api.jl restated here."""
import types

import numpy as np
import pytest

from conftest import fem

pp = fem.postprocess


def written(tmp_path, fn):
    path = tmp_path / "out.vtk"
    fn(str(path))
    return path.read_text()


def tri():
    return fem.VtkMesh(np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]), [[1, 2, 3]])


def test_writes_a_legacy_ascii_unstructured_grid(tmp_path):
    text = written(tmp_path, lambda p: fem.write_vtk(p, tri(), point_data={"T": [1.0, 2.0, 3.0]},
                                                     cell_data={"Q": [4.0]}, title="tiny"))
    for s in ("# vtk DataFile Version 3.0", "tiny", "DATASET UNSTRUCTURED_GRID", "POINTS 3 float",
              "CELLS 1 4", "CELL_TYPES 1\n5", "POINT_DATA 3", "SCALARS T float 1", "CELL_DATA 1",
              "SCALARS Q float 1"):
        assert s in text


def test_high_order_triangle_is_written_by_its_corners(tmp_path):
    coords = np.array([[0, 0], [1, 0], [0, 1], [0.5, 0], [0.5, 0.5], [0, 0.5]], dtype=float)
    mesh = fem.VtkMesh(coords, [[1, 2, 3, 4, 5, 6]])
    text = written(tmp_path, lambda p: fem.write_vtk(p, mesh, point_data={"marker": np.arange(10.0, 16.0)}))
    assert "POINTS 3 float" in text
    assert "CELLS 1 4\n3 0 1 2" in text
    assert "SCALARS marker float 1\nLOOKUP_TABLE default\n10.0\n11.0\n12.0" in text


def test_hex27_mixed_mesh_writes_its_velocity_cells(tmp_path):
    mesh = fem.structured_mixed_mesh(3, (1, 1, 1))
    text = written(tmp_path, lambda p: fem.write_vtk(p, mesh))
    assert "POINTS 8 float" in text
    assert "CELLS 1 9\n8 " in text
    assert "CELL_TYPES 1\n12" in text


def test_tuple_fields_are_vectors(tmp_path):
    text = written(tmp_path, lambda p: fem.write_vtk(p, tri(), point_data={"v": ([1.0, 2.0, 3.0], [4.0, 5.0, 6.0])},
                                                     cell_data={"f": ([1.0], [2.0], [3.0])}))
    # a plane vector pads the third component
    assert "VECTORS v float\n1.0 4.0 0.0\n2.0 5.0 0.0\n3.0 6.0 0.0" in text
    assert "VECTORS f float\n1.0 2.0 3.0" in text
    with pytest.raises(ValueError, match="must hold 2 or 3"):
        fem.write_vtk(str(tmp_path / "x.vtk"), tri(), point_data={"v": ([1.0, 2.0, 3.0],)})
    with pytest.raises(ValueError):
        fem.write_vtk(str(tmp_path / "x.vtk"), tri(), point_data={"v": ([1.0, 2.0, 3.0], [1.0, 2.0])})


def test_six_component_tuples_are_symmetric_tensors(tmp_path):
    text = written(tmp_path, lambda p: fem.write_vtk(p, tri(), cell_data={"t": ([1.0], [2.0], [3.0], [4.0], [5.0], [6.0])}))
    assert "TENSORS t float\n1.0 4.0 5.0\n4.0 2.0 6.0\n5.0 6.0 3.0" in text


def test_field_lengths_are_validated(tmp_path):
    with pytest.raises(ValueError):
        fem.write_vtk(str(tmp_path / "x.vtk"), tri(), point_data={"bad": [1.0, 2.0]})
    with pytest.raises(ValueError):
        fem.write_vtk(str(tmp_path / "x.vtk"), tri(), cell_data={"bad": [1.0, 2.0]})


def test_stokes_writer_2d_on_a_continuous_pressure_triangle(tmp_path):
    coords = np.array([[0, 0], [1, 0], [0, 1], [0.5, 0], [0.5, 0.5], [0, 0.5]], dtype=float)
    mesh = types.SimpleNamespace(dim=2, coords=coords, el2n=np.array([[1, 2, 3, 4, 5, 6]]),
                                 el2nP=np.array([[1, 2, 3]]), pressure_continuous=True)
    post = pp.Diagnostics2D(*[[float(i)] for i in range(1, 11)])
    advected = np.array([[2.0, 0.0], [0.0, 2.0], [0.0, 0.0], [1.0, 1.0], [0.0, 1.0], [1.0, 0.0]])
    text = written(tmp_path, lambda p: fem.write_stokes_vtk(p, mesh, advected, [[1, 2, 3]], [[1, 2, 3]],
                                                            [10.0, 20.0, 30.0], (np.arange(1.0, 7.0),
                                                                                 np.arange(2.0, 8.0)),
                                                            post, Q=[4.0, 5.0, 6.0]))
    for s in ("POINT_DATA 3", "2.0 0.0", "SCALARS P float 1", "SCALARS Vx float 1", "VECTORS V float",
              "CELL_DATA 1", "SCALARS strain_xx float 1", "SCALARS tau_II float 1", "SCALARS Q float 1"):
        assert s in text


def test_stokes_writer_3d_writes_vectors_and_tensors(tmp_path):
    mesh = fem.structured_mixed_mesh(3, (1, 1, 1))
    velocity = tuple(np.full(mesh.nnodes, float(c)) for c in (1, 2, 3))
    post = pp.Diagnostics3D(*[[float(i)] for i in range(1, 15)])
    text = written(tmp_path, lambda p: fem.write_stokes_vtk(p, mesh, mesh.coords, mesh.el2nP, mesh.dofsP,
                                                            np.ones(mesh.nnodesP), velocity, post))
    assert "POINT_DATA 8" in text
    assert "VECTORS velocity float\n1.0 2.0 3.0" in text
    assert "SCALARS P float 1" in text
    zs = text.split("SCALARS z float 1\nLOOKUP_TABLE default\n")[1].split("\n")[:8]
    assert sorted(float(z) for z in zs) == [0.0] * 4 + [1.0] * 4
    assert "TENSORS tau float\n8.0 11.0 12.0\n11.0 9.0 13.0\n12.0 13.0 10.0" in text
    assert "TENSORS strain float\n1.0 4.0 5.0\n4.0 2.0 6.0\n5.0 6.0 3.0" in text
    assert "SCALARS tau_II float 1" in text


def parse_vtk(text):
    lines = [ln.strip() for ln in text.split("\n") if ln.strip()]
    out = dict(points=[], cells=[], cell_types=[], point_data={}, cell_data={})
    npts = ncells = 0
    section = None
    i = 0
    while i < len(lines):
        f = lines[i].split()
        if f[0] == "POINTS":
            npts = int(f[1])
            out["points"] = [[float(x) for x in lines[i + k].split()] for k in range(1, npts + 1)]
            i += npts
        elif f[0] == "CELLS":
            ncells = int(f[1])
            out["cells"] = [[int(x) for x in lines[i + k].split()][1:] for k in range(1, ncells + 1)]
            i += ncells
        elif f[0] == "CELL_TYPES":
            n = int(f[1])
            out["cell_types"] = [int(lines[i + k]) for k in range(1, n + 1)]
            i += n
        elif f[0] == "POINT_DATA":
            section = out["point_data"]
        elif f[0] == "CELL_DATA":
            section = out["cell_data"]
        elif f[0] == "SCALARS":
            n = npts if section is out["point_data"] else ncells
            section[f[1]] = [float(lines[i + 1 + k]) for k in range(1, n + 1)]
            i += 1 + n
        i += 1
    return out


def test_round_trip_of_a_triangle_pair(tmp_path):
    mesh = fem.VtkMesh(np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0]]), [[1, 2, 3], [2, 4, 3]])
    T, Q = [1.0, 2.0, 4.0, 8.0], [7.0, 9.0]
    vtk = parse_vtk(written(tmp_path, lambda p: fem.write_vtk(p, mesh, point_data={"T": T}, cell_data={"Q": Q},
                                                              title="pair")))
    assert [p[:2] for p in vtk["points"]] == [[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0]]
    assert all(p[2] == 0.0 for p in vtk["points"])
    assert vtk["cells"] == [[0, 1, 2], [1, 3, 2]]
    assert vtk["cell_types"] == [5, 5]
    assert vtk["point_data"]["T"] == T
    assert vtk["cell_data"]["Q"] == Q


def test_unsupported_cell_layouts_are_rejected(tmp_path):
    for dim, n, what in ((1, 4, "line"), (2, 5, "2D"), (3, 5, "3D")):
        with pytest.raises(ValueError, match=f"cannot write VTK {what} cells with {n} local nodes"):
            pp.vtk_corner_rows(dim, n)
    mesh = fem.VtkMesh(np.zeros((6, 2)), [[1, 2, 3, 4, 5]])
    with pytest.raises(ValueError, match="cannot write VTK 2D cells with 5 local nodes"):
        fem.write_vtk(str(tmp_path / "x.vtk"), mesh)


def test_cell_stresses_project_to_node_means():
    el2n = np.array([[1, 2, 3], [2, 3, 4]])
    post = pp.Diagnostics2D(*([np.zeros(2)] * 5 + [np.array([1.0, 3.0]), np.array([2.0, 4.0]), np.zeros(2),
                                                    np.array([-1.0, 1.0]), np.zeros(2)]))
    tau_old = [np.full(5, 9.0) for _ in range(3)]
    fem.update_old_stress_from_cells(tau_old, post, el2n, 5)
    np.testing.assert_array_equal(tau_old[0], [1.0, 2.0, 2.0, 3.0, 0.0])
    np.testing.assert_array_equal(tau_old[1], [2.0, 3.0, 3.0, 4.0, 0.0])
    np.testing.assert_array_equal(tau_old[2], [-1.0, 0.0, 0.0, 1.0, 0.0])
