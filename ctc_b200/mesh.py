"""Membrane meshes: OFF input and the synthetic red-blood-cell template.

* ``read_off`` reads the reference's mesh files (src/io/mesh_read/imp/main.h
  reads ``OFF / nv nt ne / vertices / 3 i j k`` faces).
* ``icosphere`` + ``evans_fung`` build the RBC template of the benchmark
  configurations: a level-3 subdivided icosahedron (642 vertices, 1280
  triangles, valence 5 and 6, the topology of the reference's
  src/data/cells/rbc/642.off) mapped onto the biconcave Evans-Fung shape
  (Evans & Fung, Microvasc. Res. 4:335, 1972): thickness
  h(r) = sqrt(1-(r/R)^2) (C0 + C2 (r/R)^2 + C4 (r/R)^4), R = D/2,
  C0 = 0.81, C2 = 7.83, C4 = -4.39 for D = 7.82.
"""
import numpy as np


def read_off(path):
    """Returns (vertices float32 (nv,3), triangles int32 (nt,3))."""
    with open(path) as f:
        toks = f.read().split()
    if toks[0] != "OFF":
        raise ValueError("not an OFF file: %s" % path)
    nv, nt = int(toks[1]), int(toks[2])
    k = 4
    vert = np.array(toks[k:k + 3 * nv], dtype=np.float64).astype(np.float32).reshape(nv, 3)
    k += 3 * nv
    tri = np.zeros((nt, 3), np.int32)
    for t in range(nt):
        if int(toks[k]) != 3:
            raise ValueError("only triangles are supported")
        tri[t] = [int(toks[k + 1]), int(toks[k + 2]), int(toks[k + 3])]
        k += 4
    return vert, tri


def icosphere(level=3):
    """Unit icosphere by repeated edge-midpoint subdivision; outward-oriented."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
         (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
         (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
         (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, float) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(level):
        mid = {}

        def midpoint(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                p = verts[a] + verts[b]
                verts.append(p / np.linalg.norm(p))
                mid[key] = len(verts) - 1
            return mid[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.array(verts)
    F = np.array(faces, np.int32)
    # outward orientation: (b-a) x (c-a) . a > 0
    n = np.cross(V[F[:, 1]] - V[F[:, 0]], V[F[:, 2]] - V[F[:, 0]])
    flip = (n * V[F[:, 0]]).sum(1) < 0
    F[flip] = F[flip][:, [0, 2, 1]]
    return V, F


def evans_fung(V, D=7.82, C0=0.81, C2=7.83, C4=-4.39):
    """Map unit-sphere points onto the biconcave Evans-Fung surface of diameter D."""
    R = 0.5 * D
    x, y, z = V[:, 0], V[:, 1], V[:, 2]
    rho2 = np.clip(x * x + y * y, 0.0, 1.0)
    out = np.empty_like(V)
    out[:, 0] = R * x
    out[:, 1] = R * y
    out[:, 2] = 0.5 * z * (C0 + C2 * rho2 + C4 * rho2 * rho2)
    return out


def rbc_template(D=7.82, level=3):
    """(vertices float32 (642,3), triangles int32 (1280,3)) centred at 0."""
    V, F = icosphere(level)
    X = evans_fung(V, D)
    X -= X.mean(0)
    return X.astype(np.float32), F


def area_volume(X, F):
    """Total area and enclosed volume of a closed, outward-oriented mesh (double)."""
    X = np.asarray(X, np.float64)
    a, b, c = X[F[:, 0]], X[F[:, 1]], X[F[:, 2]]
    area = 0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1).sum()
    vol = (np.cross(a, b) * c).sum() / 6.0
    return area, vol


def random_rotation(rng):
    """Uniform random rotation matrix (quaternion method)."""
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
