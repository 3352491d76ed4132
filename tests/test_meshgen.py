"""Host-side mesh generation and dof numbering (CPU)."""

import os

import numpy as np
import pytest

from conftest import GOLDEN
from pdekit_b200 import meshgen
from golden_io import load_golden


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_equidistant_nodes_match_reference(p):
    case = {1: "adv_p1_lda", 2: "burgers_p2_b", 3: "burgers_p3_b"}.get(p)
    nodes = meshgen.equidist_triag_nodes(p)
    assert nodes.shape[0] == (p + 1) * (p + 2) // 2
    if case:
        _, a, _ = load_golden(os.path.join(GOLDEN, case))
        np.testing.assert_array_equal(nodes, a["sol_nodes"])


def test_unit_square_counts_and_orientation():
    m = meshgen.unit_square_tri(64, 0.2, seed=3)
    assert m.cells.shape == (8192, 3)
    assert m.coords.shape == (4225, 2)
    X = m.coords[m.cells]
    area2 = (X[:, 1, 0] - X[:, 0, 0]) * (X[:, 2, 1] - X[:, 0, 1]) - \
            (X[:, 1, 1] - X[:, 0, 1]) * (X[:, 2, 0] - X[:, 0, 0])
    assert (area2 > 0).all()
    np.testing.assert_allclose(area2.sum() / 2, 1.0, rtol=1e-12)


@pytest.mark.parametrize("p", [2, 3])
def test_clone_continuous_shares_dofs(p):
    m = meshgen.unit_square_tri(5, 0.1, seed=1)
    conn, nsol, xy = meshgen.clone_continuous_tri(m, p)
    n = 5 * p + 1
    assert nsol == n * n
    assert len(np.unique(conn)) == nsol
    # every dof's coordinate is consistent between the cells that share it
    ref = meshgen.equidist_triag_nodes(p)
    lam = np.stack([1 - (ref[:, 0] + 1) / 2 - (ref[:, 1] + 1) / 2, (ref[:, 0] + 1) / 2,
                    (ref[:, 1] + 1) / 2], 1)
    per_cell = np.einsum("nk,ckd->cnd", lam, m.coords[m.cells])
    np.testing.assert_allclose(per_cell, xy[conn], atol=1e-14)


def test_gmsh_roundtrip_header(tmp_path):
    m = meshgen.unit_square_tri(3, 0.0)
    f = tmp_path / "m.msh"
    meshgen.write_gmsh22(str(f), m)
    text = f.read_text()
    assert text.startswith("$MeshFormat\n2.2 0 8\n")
    assert '"bottom"' in text and "$EndElements" in text
