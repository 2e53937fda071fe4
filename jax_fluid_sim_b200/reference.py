"""Reference-element tables for the device plan.

Nodal Lagrange bases are built from a Legendre-product modal basis and the
inverse generalised Vandermonde matrix on the reference's node sets, for the
polynomial spaces the reference uses (hexahedron Q_P, wedge P_P(x,y) x P_P(z),
tetrahedron P_P).  The nodes, their order and the quadrature rules are part of
the state-layout contract and follow ``hybrid/elements.py:35-128,199-403`` and
``hybrid/geometry.py:48-89`` of superboss2300/jax-fluid-sim.
"""

from functools import lru_cache

import numpy as np

CORNERS = {
    "tetra": np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float),
    "wedge": np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [0, 1, 1]], float),
    "hexahedron": np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                            [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float),
}
LOCAL_FACES = {
    "tetra": ((0, 2, 1), (0, 1, 3), (1, 2, 3), (2, 0, 3)),
    "wedge": ((0, 2, 1), (3, 4, 5), (0, 1, 4, 3), (1, 2, 5, 4), (2, 0, 3, 5)),
    "hexahedron": ((0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7)),
}
TYPE_ID = {"hexahedron": 0, "wedge": 1, "tetra": 2}
FACE_TYPE_ID = {"triangle": 0, "quad": 1}


def _line_nodes(degree):
    return {1: (0.0, 1.0), 2: (0.0, 1.0, 0.5), 3: (0.0, 1.0, 1.0 / 3.0, 2.0 / 3.0)}[degree]


def _triangle_nodes(degree):
    t = 1.0 / 3.0
    return {
        1: [(0, 0), (1, 0), (0, 1)],
        2: [(0, 0), (1, 0), (0, 1), (.5, 0), (.5, .5), (0, .5)],
        3: [(0, 0), (1, 0), (0, 1), (t, 0), (2 * t, 0), (2 * t, t), (t, 2 * t), (0, 2 * t), (0, t), (t, t)],
    }[degree]


def nodes(element_type, degree):
    if degree == 1:
        return CORNERS[element_type].copy()
    if element_type == "hexahedron":
        line = _line_nodes(degree)
        return np.array([[x, y, z] for z in line for y in line for x in line], float)
    if element_type == "wedge":
        line = _line_nodes(degree)
        return np.array([[x, y, z] for z in line for x, y in _triangle_nodes(degree)], float)
    t = 1.0 / 3.0
    if degree == 2:
        pts = [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [.5, 0, 0], [0, .5, 0], [0, 0, .5],
               [.5, .5, 0], [.5, 0, .5], [0, .5, .5]]
    else:
        pts = [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]]
        for a, b in ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)):
            ca, cb = CORNERS["tetra"][a], CORNERS["tetra"][b]
            pts += [list((2 * ca + cb) / 3.0), list((ca + 2 * cb) / 3.0)]
        for a, b, c in ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)):
            pts.append(list((CORNERS["tetra"][a] + CORNERS["tetra"][b] + CORNERS["tetra"][c]) / 3.0))
    return np.asarray(pts, float)


def _modal_exponents(element_type, degree):
    r = range(degree + 1)
    if element_type == "hexahedron":
        return [(a, b, c) for c in r for b in r for a in r]
    if element_type == "wedge":
        return [(a, b, c) for c in r for b in r for a in r if a + b <= degree]
    return [(a, b, c) for c in r for b in r for a in r if a + b + c <= degree]


def _legendre(n, t):
    """P_n(2t-1) and its t-derivative, for arrays t."""
    s = 2.0 * t - 1.0
    p0, p1 = np.ones_like(s), s
    d0, d1 = np.zeros_like(s), np.ones_like(s)
    if n == 0:
        return p0, d0 * 2.0
    for k in range(1, n):
        p0, p1 = p1, ((2 * k + 1) * s * p1 - k * p0) / (k + 1)
        d0, d1 = d1, ((2 * k + 1) * (p0 + s * d1) - k * d0) / (k + 1)
    return p1, 2.0 * d1


def _modal(element_type, degree, points):
    pts = np.asarray(points, float).reshape(-1, 3)
    exps = _modal_exponents(element_type, degree)
    V = np.empty((len(pts), len(exps)))
    G = np.empty((len(pts), len(exps), 3))
    cache = {}
    for axis in range(3):
        for n in range(degree + 1):
            cache[axis, n] = _legendre(n, pts[:, axis])
    for k, e in enumerate(exps):
        (px, dx), (py, dy), (pz, dz) = (cache[0, e[0]], cache[1, e[1]], cache[2, e[2]])
        V[:, k] = px * py * pz
        G[:, k, 0] = dx * py * pz
        G[:, k, 1] = px * dy * pz
        G[:, k, 2] = px * py * dz
    return V, G


@lru_cache(maxsize=None)
def _coefficients(element_type, degree):
    V, _ = _modal(element_type, degree, nodes(element_type, degree))
    return np.linalg.inv(V)


def basis(element_type, degree, points):
    points = np.asarray(points, float)
    V, _ = _modal(element_type, degree, points)
    out = V @ _coefficients(element_type, degree)
    return out.reshape(points.shape[:-1] + (out.shape[-1],))


def basis_gradients(element_type, degree, points):
    points = np.asarray(points, float)
    _, G = _modal(element_type, degree, points)
    out = np.einsum("pkd,ki->pid", G, _coefficients(element_type, degree))
    return out.reshape(points.shape[:-1] + out.shape[-2:])


def gauss01(order):
    x, w = np.polynomial.legendre.leggauss(order)
    return 0.5 * (x + 1.0), 0.5 * w


def volume_quadrature(element_type, degree):
    """Collapsed (Duffy) Gauss rules at P2/P3, small rules at P1 (elements.py:60-128)."""
    if degree in (2, 3):
        g, w = gauss01(5 if (degree == 3 or element_type != "hexahedron") else 3)
        A, B, C = np.meshgrid(g, g, g, indexing="ij")
        WA, WB, WC = np.meshgrid(w, w, w, indexing="ij")
        a, b, c = A.ravel(), B.ravel(), C.ravel()
        wa, wb, wc = WA.ravel(), WB.ravel(), WC.ravel()
        if element_type == "tetra":       # a outer, b, c inner
            pts = np.stack([a, (1 - a) * b, (1 - a) * (1 - b) * c], 1)
            wts = wa * wb * wc * (1 - a) ** 2 * (1 - b)
        elif element_type == "wedge":     # z outer, a, b inner
            z, aa, bb = a, b, c
            pts = np.stack([aa, (1 - aa) * bb, z], 1)
            wts = wb * wc * wa * (1 - aa)
        else:                             # z outer, y, x inner
            pts = np.stack([c, b, a], 1)
            wts = wc * wb * wa
        return pts, wts
    if element_type == "tetra":
        a, b = 0.5854101966249685, 0.1381966011250105
        return np.array([[b, b, b], [a, b, b], [b, a, b], [b, b, a]]), np.full(4, 1.0 / 24.0)
    lp = 0.5 * (1.0 + np.array([-1.0, 1.0]) / np.sqrt(3.0))
    if element_type == "wedge":
        tri = np.array([[1 / 6, 1 / 6], [2 / 3, 1 / 6], [1 / 6, 2 / 3]])
        pts = np.array([[x, y, z] for z in lp for x, y in tri])
        return pts, np.full(6, 1.0 / 12.0)
    pts = np.array([[x, y, z] for z in lp for y in lp for x in lp])
    return pts, np.full(8, 0.125)


def face_quadrature(face_type, degree):
    """(shape values on the face corners, weights summing to 1): geometry.py:48-89."""
    if face_type == "triangle" and degree == 1:
        s = np.array([[2 / 3, 1 / 6, 1 / 6], [1 / 6, 2 / 3, 1 / 6], [1 / 6, 1 / 6, 2 / 3]])
        return s, np.full(3, 1.0 / 3.0)
    if face_type == "triangle":
        g, w = gauss01(4 if degree <= 2 else 5)
        A, B = np.meshgrid(g, g, indexing="ij")
        WA, WB = np.meshgrid(w, w, indexing="ij")
        x, y = A.ravel(), (1 - A.ravel()) * B.ravel()
        return np.stack([1 - x - y, x, y], 1), 2.0 * WA.ravel() * WB.ravel() * (1 - A.ravel())
    g, w = gauss01({1: 2, 2: 3, 3: 4}[degree])
    V, U = np.meshgrid(g, g, indexing="ij")
    WV, WU = np.meshgrid(w, w, indexing="ij")
    u, v = U.ravel(), V.ravel()
    return np.stack([(1 - u) * (1 - v), u * (1 - v), u * v, (1 - u) * v], 1), WU.ravel() * WV.ravel()


class RefElement:
    def __init__(self, element_type, degree):
        if degree not in (1, 2, 3):
            raise ValueError("Only P1, P2, and P3 are currently implemented")
        self.element_type, self.degree = element_type, degree
        self.nodes = nodes(element_type, degree)
        self.points, self.weights = volume_quadrature(element_type, degree)
        self.B = basis(element_type, degree, self.points)
        self.dB = basis_gradients(element_type, degree, self.points)
        self.mass = (self.B * self.weights[:, None]).T @ self.B
        self.np = len(self.nodes)
        self.nq = len(self.points)

    def basis(self, points):
        return basis(self.element_type, self.degree, points)

    def basis_gradients(self, points):
        return basis_gradients(self.element_type, self.degree, points)
