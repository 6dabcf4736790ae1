"""Element colouring (color_mesh_greedy / generate_element_groups,
src/mesh/coloring.jl:26-81): host code of libfemtools_b200, no GPU needed."""
import numpy as np
import pytest

from conftest import fem


def greedy_reference(el2n, nnodes):
    """The greedy rule of coloring.jl:26-50 as plain Python loops."""
    nels = len(el2n)
    n2el = [[] for _ in range(nnodes)]
    for e in range(nels):
        for n in el2n[e]:
            n2el[n - 1].append(e)
    colors = [0] * nels
    for e in range(nels):
        used = {colors[j] for n in el2n[e] for j in n2el[n - 1] if colors[j] != 0}
        c = 1
        while c in used:
            c += 1
        colors[e] = c
    return np.array(colors, dtype=np.int32)


def valid(el2n, colors):
    for c in range(1, colors.max() + 1):
        nodes = el2n[colors == c].ravel()
        if len(np.unique(nodes)) != len(nodes):
            return False
    return True


def test_known_answers():
    # test/test_mesh.jl:200-226: six quadratic line elements alternate 1, 2
    el2n = np.array([[2 * e + 1, 2 * e + 2, 2 * e + 3] for e in range(6)], dtype=np.int32)
    assert fem.color_mesh(el2n, 13).tolist() == [1, 2, 1, 2, 1, 2]
    # coloring.jl:13-24: the four cells of a 2 × 2 mesh share the centre node
    mesh = fem.structured_mixed_mesh(2, (2, 2))
    assert fem.color_mesh(mesh).tolist() == [1, 2, 3, 4]


@pytest.mark.parametrize("dim,n", [(3, (4, 3, 5)), (2, (7, 5))])
def test_structured_meshes(dim, n):
    mesh = fem.structured_mixed_mesh(dim, n)
    colors = fem.color_mesh(mesh)
    assert valid(mesh.el2n, colors)
    assert colors.max() == 2 ** dim
    np.testing.assert_array_equal(colors, greedy_reference(mesh.el2n, mesh.nnodes))


def test_permuted_elements_match_the_greedy_rule():
    mesh = fem.structured_mixed_mesh(3, (3, 3, 3))
    perm = np.random.default_rng(5).permutation(mesh.nels)
    el2n = mesh.el2n[perm]
    colors = fem.color_mesh(el2n, mesh.nnodes)
    assert valid(el2n, colors)
    np.testing.assert_array_equal(colors, greedy_reference(el2n, mesh.nnodes))


def test_groups():
    colors = np.array([2, 1, 3, 1, 2, 2], dtype=np.int32)
    g = fem.generate_element_groups(colors)
    assert g.ncolors == 3
    assert g.offsets.tolist() == [0, 2, 5, 6]
    assert [g.group(c).tolist() for c in (1, 2, 3)] == [[2, 4], [1, 5, 6], [3]]


def test_rejects_bad_input():
    with pytest.raises(fem._abi.FemB200Error):
        fem.color_mesh(np.array([[1, 2, 9]], dtype=np.int32), 3)
    with pytest.raises(fem._abi.FemB200Error):
        fem.generate_element_groups(np.array([1, 0, 2], dtype=np.int32))
