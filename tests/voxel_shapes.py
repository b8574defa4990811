"""Closed triangle surfaces with known insides for the voxeliser tests, and
STL writers (binary and ASCII).  Triangles are (ntri, 9) arrays, outward
counter-clockwise."""
import numpy as np


def box(lo, hi):
    (x0, y0, z0), (x1, y1, z1) = lo, hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]])
    f = [(0, 2, 1), (0, 3, 2), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4),
         (1, 2, 6), (1, 6, 5), (2, 3, 7), (2, 7, 6), (3, 0, 4), (3, 4, 7)]
    return np.array([np.concatenate([v[a], v[b], v[c]]) for a, b, c in f])


def octahedron(c, r):
    c = np.asarray(c, float)
    v = [c + d for d in r * np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1],
                                      [0, 0, -1]])]
    f = [(0, 2, 4), (2, 1, 4), (1, 3, 4), (3, 0, 4), (2, 0, 5), (1, 2, 5), (3, 1, 5), (0, 3, 5)]
    return np.array([np.concatenate([v[a], v[b], v[cc]]) for a, b, cc in f])


def icosphere(c, R, subdiv=3):
    t = (1 + 5 ** 0.5) / 2
    v = [np.array(p, float) for p in [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0),
                                       (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
                                       (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]]
    v = [p / np.linalg.norm(p) for p in v]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
         (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
         (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache, nf = {}, []

        def mid(a, b):
            k = (min(a, b), max(a, b))
            if k not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[k] = len(v) - 1
            return cache[k]

        for a, b, cc in f:
            ab, bc, ca = mid(a, b), mid(b, cc), mid(cc, a)
            nf += [(a, ab, ca), (b, bc, ab), (cc, ca, bc), (ab, bc, ca)]
        f = nf
    c = np.asarray(c, float)
    return np.array([np.concatenate([c + R * v[a], c + R * v[b], c + R * v[cc]])
                     for a, b, cc in f])


def torus(c, R, r, nu=48, nv=24):
    c = np.asarray(c, float)
    u = np.linspace(0, 2 * np.pi, nu, endpoint=False)
    w = np.linspace(0, 2 * np.pi, nv, endpoint=False)

    def p(i, j):
        a, b = u[i % nu], w[j % nv]
        return c + np.array([(R + r * np.cos(b)) * np.cos(a), (R + r * np.cos(b)) * np.sin(a),
                             r * np.sin(b)])

    tris = []
    for i in range(nu):
        for j in range(nv):
            p00, p10, p11, p01 = p(i, j), p(i + 1, j), p(i + 1, j + 1), p(i, j + 1)
            tris.append(np.concatenate([p00, p10, p11]))
            tris.append(np.concatenate([p00, p11, p01]))
    return np.array(tris)


def write_stl_binary(path, tri):
    tri = np.asarray(tri, np.float32).reshape(-1, 9)
    rec = np.zeros(len(tri), np.dtype([("n", "<f4", 3), ("v", "<f4", 9), ("a", "<u2")]))
    rec["v"] = tri
    with open(path, "wb") as f:
        f.write(b"\0" * 80)
        f.write(np.uint32(len(tri)).tobytes())
        f.write(rec.tobytes())


def write_stl_ascii(path, tri):
    with open(path, "w") as f:
        f.write("solid s\n")
        for t in np.asarray(tri).reshape(-1, 3, 3):
            f.write("facet normal 0 0 0\n outer loop\n")
            for p in t:
                f.write("  vertex %.17g %.17g %.17g\n" % tuple(p))
            f.write(" endloop\nendfacet\n")
        f.write("endsolid s\n")
