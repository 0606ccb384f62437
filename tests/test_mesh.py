"""Mesh generators and mesh I/O (host code, no GPU)."""
import os
import tempfile

import numpy as np
import pytest

import multigridsoftbody_b200 as mg


def _dets(m):
    P = m.positions.astype(np.float64)
    T = m.tets
    D = np.stack([P[T[:, 1]] - P[T[:, 0]], P[T[:, 2]] - P[T[:, 0]], P[T[:, 3]] - P[T[:, 0]]], axis=2)
    return np.linalg.det(D)


@pytest.mark.parametrize("dims,V,T", [((4, 40, 4), 1025, 3840), ((12, 120, 12), 20449, 103680),
                                      ((24, 240, 24), 150625, 829440)])
def test_box_counts(lib, dims, V, T):
    m = mg.box_mesh(*dims)
    assert (m.num_verts, m.num_tets) == (V, T)
    assert m.grid_dims == dims


def test_box_volume_and_orientation(lib):
    m = mg.box_mesh(4, 40, 4)
    d = _dets(m)
    assert (d > 0).all()
    assert abs(d.sum() / 6.0 - 80.0) < 1e-9


def test_kuhn_valence(lib):
    m = mg.box_mesh(4, 6, 4)
    nb = [set() for _ in range(m.num_verts)]
    for t in m.tets:
        for a in t:
            nb[a].update(int(b) for b in t if b != a)
    # interior vertex (i=2, j=3, k=2) of a Freudenthal grid has 14 neighbours
    vid = 2 + 5 * (2 + 5 * 3)
    assert len(nb[vid]) == 14


def test_surface_matches_reference(lib, golden_cpu):
    """Boundary faces + opposite vertex equal SoftObject::TetFaceExtraction's, in order."""
    tets = golden_cpu["surf_tets"]
    b = mg.box_mesh(2, 8, 3)
    assert np.array_equal(b.tets, tets)
    mg.extract_surface(b)
    assert np.array_equal(b.tris, golden_cpu["surf_tris"])
    assert np.array_equal(b.tri_opposite, golden_cpu["surf_opp"])


def test_surface_count_box(lib):
    m = mg.extract_surface(mg.box_mesh(4, 40, 4))
    assert m.tris.shape == (1344, 3)   # 2*(4*40 + 4*40 + 4*4) quads, 2 triangles each


def test_msh_reader_matches_reference(lib, golden_cpu):
    """gmsh 2.2 reader equals SoftObject::ReadFromFile on the same file."""
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "g.msh")
        with open(p, "wb") as f:
            f.write(golden_cpu["msh_text"].tobytes())
        m = mg.read_msh(p)
    assert np.array_equal(m.tets, golden_cpu["msh_tets"])
    assert np.allclose(m.positions, golden_cpu["msh_pos"], rtol=0, atol=1e-6)
    mg.extract_surface(m)
    assert np.array_equal(m.tris, golden_cpu["msh_tris"])
    assert np.array_equal(m.tri_opposite, golden_cpu["msh_opp"])


def test_msh_reader_errors(lib):
    with pytest.raises(mg.MgsbError):
        mg.read_msh("/nonexistent/file.msh")
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "bad.msh")
        with open(p, "w") as f:
            f.write("$Nodes\n2\n1 0 0 0\n2 1 0 0\n$EndNodes\n$Elements\n1\n1 4 2 0 1 1 2 3 9\n$EndElements\n")
        with pytest.raises(mg.MgsbError):
            mg.read_msh(p)


def test_value_noise(lib):
    a = mg.value_noise(0.3, 1.7, -2.2, 2.0, 3)
    assert a == mg.value_noise(0.3, 1.7, -2.2, 2.0, 3)
    assert a != mg.value_noise(0.3, 1.7, -2.2, 2.0, 4)
    # lattice values in [-1, 1), interpolation keeps the range
    xs = np.linspace(-8, 8, 37)
    vals = [mg.value_noise(x, 0.5 * x, -0.25 * x, 2.0, 3) for x in xs]
    assert max(abs(v) for v in vals) <= 1.0
    # continuity across a lattice plane
    assert abs(mg.value_noise(2.0 - 1e-9, 0.3, 0.1, 2.0, 3) - mg.value_noise(2.0 + 1e-9, 0.3, 0.1, 2.0, 3)) < 1e-6


def test_blob_config(lib):
    m = mg.blob_mesh()   # 64x32x48 voxels at 0.25, ellipsoid (6,3,4), amp 0.15, period 2, seed 3
    # ellipsoid volume 4/3*pi*6*3*4 = 301.6 m^3 -> ~19.3k voxels of 0.25^3 -> ~116k tets
    assert 100_000 < m.num_tets < 135_000
    assert m.num_tets % 6 == 0
    assert (_dets(m) > 0).all()
    m2 = mg.blob_mesh()
    assert np.array_equal(m.tets, m2.tets)
    used = np.zeros(m.num_verts, bool)
    used[m.tets.reshape(-1)] = True
    assert used.all()


def test_batch_sizes_seed11(lib):
    rng = np.random.default_rng(11)
    ns = rng.integers(2, 9, size=256)
    V = sum((n + 1) * (10 * n + 1) * (n + 1) for n in ns)
    T = sum(6 * n * 10 * n * n for n in ns)
    assert 300_000 < V < 1_000_000 and 1_000_000 < T < 5_000_000
