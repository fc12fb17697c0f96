"""The generated marching-cubes table (dynamap_b200/mc_tables.py ->
csrc/mc_tables.h): the header matches its generator, each configuration's
triangles use exactly its cut edges, and meshes built with it are closed
and consistently oriented with normals towards positive values -- on a
sphere (Euler characteristic 2) and on random fields, whose ambiguous faces
adjacent cells must cut alike."""
import numpy as np
import pytest

from dynamap_b200 import mc_tables as mc


def test_header_matches_generator():
    with open(mc.HEADER) as f:
        assert f.read() == mc.header_text()


def test_rows_use_exactly_the_cut_edges():
    t = mc.table()
    assert t[0] == [] and t[255] == []
    for cube, tris in enumerate(t):
        below = [(cube >> k) & 1 for k in range(8)]
        cut = {e for e, (a, b) in enumerate(mc.EDGE) if below[a] != below[b]}
        assert len(tris) % 3 == 0 and len(tris) // 3 <= 5
        assert set(tris) == cut, cube
        for j in range(0, len(tris), 3):
            assert len(set(tris[j:j + 3])) == 3


def extract(field):
    """Mesh of field < 0 on a grid of unit cells: vertices keyed by their
    grid edge, triangles as vertex-key triples, positions by linear
    interpolation."""
    table = mc.table()
    n = np.array(field.shape) - 1
    corner = np.array(mc.CORNER)
    tris, pos = [], {}
    for i in range(n[0]):
        for j in range(n[1]):
            for k in range(n[2]):
                base = np.array([i, j, k])
                vals = [field[tuple(base + c)] for c in corner]
                cube = sum(1 << c for c in range(8) if vals[c] < 0)
                row = table[cube]
                for t in range(0, len(row), 3):
                    tri = []
                    for e in row[t:t + 3]:
                        a, b = mc.EDGE[e]
                        pa, pb = tuple(base + corner[a]), tuple(base + corner[b])
                        key = (min(pa, pb), max(pa, pb))
                        if key not in pos:
                            va, vb = vals[a], vals[b]
                            mu = va / (va - vb)
                            pos[key] = np.array(pa) + mu * (np.array(pb) - np.array(pa))
                        tri.append(key)
                    tris.append(tri)
    return tris, pos


def check_closed_oriented(tris):
    """Every mesh edge is walked as often in one direction as in the other
    (closed and consistently oriented; a loop's fan can put a diagonal on a
    face the neighbouring cell's fan also crosses, so an edge may bound four
    triangles)."""
    directed = {}
    for t in tris:
        for u in range(3):
            e = (t[u], t[(u + 1) % 3])
            directed[e] = directed.get(e, 0) + 1
    for (a, b), cnt in directed.items():
        assert directed.get((b, a), 0) == cnt, "an open or inconsistently oriented edge"


def test_sphere_closed_outward_genus_zero():
    g = np.arange(18, dtype=np.float64)
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    c = np.array([8.3, 8.7, 8.1])
    field = np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) - 6.2
    tris, pos = extract(field)
    assert len(tris) > 500
    check_closed_oriented(tris)
    edges = {frozenset((t[u], t[(u + 1) % 3])) for t in tris for u in range(3)}
    assert len(pos) - len(edges) + len(tris) == 2
    for t in tris:
        p0, p1, p2 = (pos[k] for k in t)
        nrm = np.cross(p1 - p0, p2 - p0)
        if np.linalg.norm(nrm) > 1e-9:
            assert np.dot(nrm, (p0 + p1 + p2) / 3 - c) > 0


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_random_fields_closed(seed):
    rng = np.random.default_rng(seed)
    field = rng.normal(size=(12, 12, 12))
    field[0, :, :] = field[-1, :, :] = 1.0  # outside at the border: closed surfaces
    field[:, 0, :] = field[:, -1, :] = 1.0
    field[:, :, 0] = field[:, :, -1] = 1.0
    tris, _ = extract(field)
    assert len(tris) > 200
    check_closed_oriented(tris)
