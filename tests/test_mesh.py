"""Mesh generators, the polyMesh reader and the geometry routine of the
library (host code) against the oracle's independent restatement."""
import numpy as np
import pytest

import golden_cases
import oracle_bind as ob
from dugks_b200 import lib as dl
from dugks_b200 import meshgen


def _check_topology(pm):
    nIF = pm.n_internal_faces
    own, nei = pm.owner[:nIF], pm.neighbour
    assert np.all(own < nei)
    assert np.all(np.lexsort((nei, own)) == np.arange(nIF))   # upper-triangular order
    g = ob.geometry(pm)
    d = g["Cf"] - g["C"][pm.owner]
    assert np.all(np.einsum("ij,ij->i", g["Sf"], d) > 0)      # normals point out of the owner
    assert np.all(g["V"] > 0)
    return g


@pytest.mark.parametrize("pm", [meshgen.cavity(7), meshgen.cube(4), meshgen.cubed_sphere(4, 3),
                                meshgen.refined_cavity(5)],
                         ids=["cavity", "cube", "sphere", "refined"])
def test_generators_and_geometry(pm):
    g = _check_topology(pm)
    p = dl.mesh_geometry(pm)
    for k in ("Cf", "Sf", "C", "V"):
        assert np.array_equal(p[k], g[k]), k
    # closed cells: the area vectors of each cell sum to zero
    s = np.zeros((pm.n_cells, 3))
    np.add.at(s, pm.owner, g["Sf"])
    np.add.at(s, pm.neighbour, -g["Sf"][: pm.n_internal_faces])
    assert np.max(np.abs(s)) < 1e-12 * np.max(np.abs(g["Sf"]))


def test_cavity_volume_and_demo_mesh():
    c = golden_cases.demo_cavity(flatten=False)
    g = _check_topology(c.mesh)
    assert abs(g["V"].sum() - 0.1) < 1e-14
    assert c.mesh.n_cells == 3600 and c.mesh.n_internal_faces == 7080
    # the generator's 60x60 cavity holds the same cells (different numbering)
    g2 = ob.geometry(meshgen.cavity(60))
    a = np.round(g["C"], 12)
    b = np.round(g2["C"], 12)
    assert np.array_equal(a[np.lexsort(a.T)], b[np.lexsort(b.T)])


def test_cubed_sphere_counts():
    pm = meshgen.cubed_sphere(24, 32, 1.12)
    assert pm.n_cells == 110592
    assert [p["nFaces"] for p in pm.patches] == [6 * 24 * 24, 6 * 24 * 24]
    r = meshgen.radial_stations(32, 1.12, 1.0, 10.0)
    assert abs(r[0] - 1) < 1e-15 and abs(r[-1] - 10) < 1e-12
    assert np.allclose(np.diff(r)[1:] / np.diff(r)[:-1], 1.12)


def test_refined_cavity_cells_and_faces():
    # n x n squares, every other one split into 2 x 2: 4 fine cells per split
    # square; an interior octagon has eight internal faces, and with front and
    # back ten faces in all
    n = 6
    pm = meshgen.refined_cavity(n)
    split = sum((i + j) % 2 == 0 for i in range(n) for j in range(n))
    assert pm.n_cells == 4 * split + (n * n - split)
    nif = pm.n_internal_faces
    internal = np.bincount(np.concatenate([pm.owner[:nif], pm.neighbour]), minlength=pm.n_cells)
    faces = np.bincount(pm.owner, minlength=pm.n_cells) + np.bincount(pm.neighbour, minlength=pm.n_cells)
    assert internal.max() == 8 and faces.max() == 10
    g = _check_topology(pm)
    assert abs(g["V"].sum() - 0.1) < 1e-14
    # the octagons keep the square's centroid
    octagon = np.nonzero(internal == 8)[0]
    c = g["C"][octagon, :2] * n
    assert np.max(np.abs(c - (np.floor(c) + 0.5))) < 1e-12
