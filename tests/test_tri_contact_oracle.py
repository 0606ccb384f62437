"""The oracle's capsule-against-surface-triangle narrow phase on CPU: the
segment-triangle distance against dense sampling, and a capsule that enters a
coarse face between its vertices, found only by the triangle test."""
import numpy as np

import multigridsoftbody_b200 as mg
from oracle.binding import Oracle, segment_triangle

from .common import beam, mg_params


def _sampled_distance(p0, p1, a, b, c, n=120):
    s = np.linspace(0.0, 1.0, n)
    seg = p0[None] + s[:, None] * (p1 - p0)[None]
    u, v = np.meshgrid(np.linspace(0, 1, n), np.linspace(0, 1, n))
    keep = (u + v) <= 1.0
    tri = a[None] + u[keep][:, None] * (b - a)[None] + v[keep][:, None] * (c - a)[None]
    d2 = ((seg[:, None, :] - tri[None, :, :]) ** 2).sum(-1)
    return float(np.sqrt(d2.min()))


def test_segment_triangle_distance_matches_sampling():
    rng = np.random.default_rng(3)
    for _ in range(60):
        a, b, c = rng.normal(size=(3, 3))
        p0, p1 = rng.normal(size=(2, 3)) * 1.5
        d, q, h = segment_triangle(p0, p1, a, b, c)
        ds = _sampled_distance(p0, p1, a, b, c)
        assert d <= ds + 1e-12                     # exact minimum: never above a sampled pair
        assert ds - d < 0.05 * (1.0 + np.abs([a, b, c, p0, p1]).max())   # and close to the sampled one
        assert abs(np.linalg.norm(q - h) - d) < 1e-9
    # a segment through the face has distance 0
    d, q, h = segment_triangle(np.array([0.2, 0.2, -1.0]), np.array([0.2, 0.2, 1.0]),
                               np.array([0.0, 0.0, 0.0]), np.array([1.0, 0.0, 0.0]), np.array([0.0, 1.0, 0.0]))
    assert d == 0.0 and np.allclose(q, [0.2, 0.2, 0.0])


def test_capsule_between_vertices_found_by_triangles_only():
    """A 2x20x2-hex beam (vertex spacing 1 across, 1 along): a capsule of radius 0.2 along x, 0.15 above
    the top face and midway between two vertex rows, is 0.29 from every vertex but 0.15 from the faces."""
    m, fixed = beam(2, 20, 2)
    p = mg_params(levels=2, gravity=(0.0, 0.0, 0.0))
    a = np.array([-3.0, 0.5, 1.15], np.float32)
    b = np.array([3.0, 0.5, 1.15], np.float32)
    flags = {}
    for tri in (False, True):
        o = Oracle(m, p)
        o.set_fixed(fixed)
        o.set_surface_contact(tri)
        o.set_capsule(a, b, 0.2)
        o.step()
        flags[tri] = np.nonzero(o.contact_flags())[0]
        x = o.positions()
        o.close()
        if tri:
            # the contact set = the vertices of the surface triangles within 0.2 of the segment (the first
            # frame's prediction is the rest shape: no gravity, no velocity)
            mg.extract_surface(m)
            want = set()
            for t in m.tris:
                d, _, _ = segment_triangle(a.astype(np.float64), b.astype(np.float64), *m.positions[t].astype(np.float64))
                if d < 0.2:
                    want.update(int(v) for v in t)
            assert sorted(want) == flags[tri].tolist()
            top = flags[tri][np.abs(m.positions[flags[tri], 2] - 1.0) < 1e-6]
            assert len(top) > 0 and x[top, 2].max() < 1.0          # the top face is pushed down
    assert len(flags[False]) == 0 and len(flags[True]) > 0
