"""Hull vertex order: the product's add_hull_from_mesh against dynamis-hull's rule.

The vertex numbering of a hull reaches the step: support scans break ties on the first vertex and
hull contacts carry vertex-index features that the warm start relays by. The reference's hull()
(crates/dynamis-hull/src/hull.rs:53-288) numbers the vertices by first appearance over its surviving
faces, after a quickhull whose seed is the live face whose first outside point lies farthest (the
last such face on ties), expanded from its farthest outside point (again the last on ties), with
visibility at 1e-6 in f32. `restated_hull` below is a third restatement of that rule, in numpy
float32 scalars (one IEEE binary32 operation each), written for this test alone; the expected orders
are pinned as literals, and the library (dyn_add_hull_from_mesh, dyn_add_hull) and the oracle
(oracle/scene.cpp) must both give them.

One departure from hull.rs, where it would not terminate: a point that already is a corner of a
face joins no outside set. Rounding can put such a corner beyond 1e-6 of a skinny face through it
(near-duplicate points); the reference's rounds then take it as the apex again and again, making
degenerate faces, and never end. The 18-point set of `LOOPING` is such a case (a hull of the
40^3 mixed pile).

Cases: the reference's own box mesh and repeated-vertex tetrahedron (crates/dynamis-hull/tests/
hull.rs:3-29,68-100), a box mesh whose first triangles leave a vertex unreferenced, and a seeded
24-point cloud on the unit sphere.
"""
import numpy as np

from dynamis_b200 import World
from oracle import oracle as O

F = np.float32


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _sub(a, b):
    return [a[0] - b[0], a[1] - b[1], a[2] - b[2]]


def _normal(p, a, b, c):
    ab, ac = _sub(p[b], p[a]), _sub(p[c], p[a])
    cr = [ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2], ab[0] * ac[1] - ab[1] * ac[0]]
    length = np.sqrt(_dot(cr, cr))
    if length < F(1e-12):
        return [F(0), F(0), F(0)]
    return [cr[0] / length, cr[1] / length, cr[2] / length]


def restated_hull(vertices, triangles):
    used = sorted({int(i) for t in triangles for i in t})
    p = [[F(x) for x in vertices[i]] for i in used]
    xmin = xmax = 0
    for i, q in enumerate(p):
        if q[0] < p[xmin][0]:
            xmin = i
        if q[0] > p[xmax][0]:
            xmax = i
    a, b = (0, len(p) - 1) if xmin == xmax else (xmin, xmax)
    d = _sub(p[b], p[a])
    lsq = _dot(d, d)
    best, c = F(-1), 0
    for i, q in enumerate(p):
        t = _dot(_sub(q, p[a]), d) / lsq if lsq > 0 else F(0)
        off = _sub(q, [p[a][k] + d[k] * t for k in range(3)])
        dist = np.sqrt(_dot(off, off))
        if dist > best:
            best, c = dist, i
    n0 = _normal(p, a, b, c)
    o0 = _dot(n0, p[a])
    best, e = F(0), 0
    for i, q in enumerate(p):
        dist = abs(_dot(n0, q) - o0)
        if dist > best:
            best, e = dist, i
    mid = [(p[a][k] + p[b][k] + p[c][k] + p[e][k]) * F(0.25) for k in range(3)]
    faces = []  # [a, b, c, normal, offset, outside, dead]

    def face(i, j, k):
        nn = _normal(p, i, j, k)
        return [i, j, k, nn, _dot(nn, p[i]), [], False]

    def height(f, q):
        return _dot(f[3], p[q]) - f[4]

    for i, j, k in ((a, b, c), (a, b, e), (a, c, e), (b, c, e)):
        f = face(i, j, k)
        if _dot(f[3], mid) - f[4] > 0:
            f[3] = [-x for x in f[3]]
            f[4] = -f[4]
            f[1], f[2] = f[2], f[1]
        faces.append(f)

    def assign(points):
        corners = {v for f in faces for v in f[:3]}
        for q in points:
            if q in corners:  # a corner of the hull is outside no face (see the module docstring)
                continue
            for f in faces:
                if not f[6] and height(f, q) > F(1e-6):
                    f[5].append(q)
                    break

    assign(range(len(p)))
    while True:
        live = [f for f in faces if not f[6] and f[5]]
        if not live:
            break
        seed = live[0]
        for f in live[1:]:
            if not (height(f, f[5][0]) < height(seed, seed[5][0])):
                seed = f
        apex = seed[5][0]
        for q in seed[5][1:]:
            if not (height(seed, q) < height(seed, apex)):
                apex = q
        visible = [f for f in faces if not f[6] and f is not seed and height(f, apex) > F(1e-6)] + [seed]
        edges = {(f[i], f[(i + 1) % 3]) for f in visible for i in range(3)}
        horizon = [(f[i], f[(i + 1) % 3]) for f in visible for i in range(3) if (f[(i + 1) % 3], f[i]) not in edges]
        pending = [q for f in visible for q in f[5]] + [apex]
        for f in visible:
            f[6] = True
        faces.extend(face(s, t, apex) for s, t in horizon)
        assign(pending)
    order = []
    for f in faces:
        if not f[6]:
            for v in f[:3]:
                if v not in order:
                    order.append(v)
    return np.array([p[v] for v in order], np.float32)


BOX = np.array([[-0.5, -0.5, -0.5], [0.5, -0.5, -0.5], [0.5, 0.5, -0.5], [-0.5, 0.5, -0.5],
                [-0.5, -0.5, 0.5], [0.5, -0.5, 0.5], [0.5, 0.5, 0.5], [-0.5, 0.5, 0.5]], np.float32)
BOX_TRIANGLES = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4], [3, 7, 6], [3, 6, 2],
                          [1, 2, 6], [1, 6, 5], [0, 4, 7], [0, 7, 3]], np.uint32)
# the box's hull vertices as indices into BOX, in the reference's order
BOX_ORDER = [0, 2, 1, 6, 7, 5, 4, 3]


def sphere_cloud(n=24, seed=11):
    v = np.random.default_rng(seed).normal(size=(n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


# the cloud's hull vertices as indices into sphere_cloud(), in the reference's order
CLOUD_ORDER = [0, 17, 12, 19, 16, 15, 1, 8, 7, 4, 22, 14, 6, 20, 3, 2, 18, 21, 10, 13, 23, 9, 5, 11]


def product_hull(vertices, triangles=None):
    world = World()
    if triangles is None:
        world.add_hull(vertices)
    else:
        world.add_hull_from_mesh(vertices, triangles)
    scene = world.export_scene()
    world.close()
    return scene["vertices"][:, :3]


def indices_of(hull_vertices, points):
    return [int(np.nonzero(np.all(points == v, axis=1))[0][0]) for v in hull_vertices]


def test_the_box_mesh_keeps_the_references_vertex_order():
    expected = BOX[BOX_ORDER]
    assert np.array_equal(restated_hull(BOX, BOX_TRIANGLES), expected)
    assert np.array_equal(product_hull(BOX, BOX_TRIANGLES), expected)
    hv, faces = O.hull_from_mesh(BOX, BOX_TRIANGLES)
    assert np.array_equal(hv, expected)
    # the reference's own assertions (hull.rs tests :68-81)
    assert len(hv) == 8 and len(faces) == 12 and faces.max() < len(hv)


def test_repeated_vertices_do_not_reach_the_hull():
    vertices = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0, 0, 0]], np.float32)
    triangles = np.array([[0, 1, 2], [0, 3, 1], [1, 3, 2], [2, 3, 0]], np.uint32)
    assert len(product_hull(vertices, triangles)) == 4
    assert len(O.hull_from_mesh(vertices, triangles)[0]) == 4


def test_only_referenced_vertices_are_hulled():
    # drop vertex 7 from every triangle: its corner leaves the hull
    keep = BOX_TRIANGLES[~np.any(BOX_TRIANGLES == 7, axis=1)]
    expected = restated_hull(BOX, keep)
    assert len(expected) == 7 and not np.any(np.all(expected == BOX[7], axis=1))
    assert np.array_equal(product_hull(BOX, keep), expected)
    assert np.array_equal(O.hull_from_mesh(BOX, keep)[0], expected)


def test_a_point_cloud_keeps_the_references_vertex_order():
    cloud = sphere_cloud()
    every = np.arange(24, dtype=np.uint32).reshape(8, 3)
    expected = cloud[CLOUD_ORDER]
    assert np.array_equal(restated_hull(cloud, every), expected)
    assert np.array_equal(product_hull(cloud), expected)
    assert np.array_equal(product_hull(cloud, every), expected)
    assert np.array_equal(O.hull_from_mesh(cloud)[0], expected)


# mixed_pile(side=40, seed=1)'s hull 183, exactly (float32): points 9 and 14 lie 1.4 mm apart
LOOPING = np.array([
    [-0.41411394, 0.37386918, -0.15936911],
    [-0.28930825, 0.011378564, -0.50283027],
    [-0.2002228, 0.4517614, 0.3041209],
    [0.1019397, 0.30704126, 0.48166484],
    [0.4823271, -0.20231423, 0.25119027],
    [-0.30184072, -0.45380613, -0.19904576],
    [0.024475537, -0.4240513, -0.39528275],
    [0.14983891, -0.35578495, -0.43316555],
    [0.16421627, 0.5316753, 0.164382],
    [0.5781241, -0.04024036, -0.02864001],
    [0.23364972, 0.5251438, 0.079365306],
    [0.1228779, 0.5505535, -0.13586348],
    [-0.049271557, -0.57807744, -0.00811153],
    [-0.55631566, -0.16173857, 0.031946458],
    [0.577242, -0.053670265, -0.02404614],
    [-0.48861164, 0.17595671, -0.25877583],
    [0.34605446, -0.06995607, 0.46045575],
    [0.13188206, 0.028266655, 0.56433606]], np.float32)


def test_near_duplicate_points_end_with_a_closed_hull():
    expected = restated_hull(LOOPING, np.arange(18, dtype=np.uint32).reshape(6, 3))
    assert np.array_equal(product_hull(LOOPING), expected)
    hv, faces = O.hull_from_mesh(LOOPING)
    assert np.array_equal(hv, expected)
    # a closed triangulation: V - E + F = 2 with every edge shared by two faces
    edges = {tuple(sorted((int(f[i]), int(f[(i + 1) % 3])))) for f in faces for i in range(3)}
    assert len(hv) - len(edges) + len(faces) == 2
