"""Reference elements: nodal Lagrange bases P1-P3, volume and face quadrature.

Oracle restatement of ``hybrid/elements.py`` and ``hybrid/geometry.py:48-89``.
Each basis function is written as a coefficient times a product of affine
factors of the reference coordinates, which gives values and gradients (by the
product rule) of exactly the polynomials the reference defines:

* line factors  ``hybrid/elements.py:214-219`` (P2, nodes 0, 1, 1/2) and
  ``:325-335`` (P3, nodes 0, 1, 1/3, 2/3);
* triangle      ``:222-231`` (P2), ``:338-358`` (P3);
* tetrahedron   ``:133-134`` (P1), ``:250-259`` (P2), ``:406-436`` (P3);
* wedge = triangle x line in z, line index outer (``:260-265``, ``:437-442``);
* hexahedron P1 in VTK corner order (``:147-157``), P2/P3 lexicographic with
  x fastest (``:266-274``, ``:443-456``).
"""

import numpy as np

# affine factor: (c, gx, gy, gz) meaning c + gx*x + gy*y + gz*z
_X = (0.0, 1.0, 0.0, 0.0)
_Y = (0.0, 0.0, 1.0, 0.0)
_Z = (0.0, 0.0, 0.0, 1.0)
_ONE_MINUS_X = (1.0, -1.0, 0.0, 0.0)
_ONE_MINUS_Y = (1.0, 0.0, -1.0, 0.0)
_ONE_MINUS_Z = (1.0, 0.0, 0.0, -1.0)


def _scale(f, a, b=0.0):
    """a*f + b for an affine factor f."""
    return (a * f[0] + b, a * f[1], a * f[2], a * f[3])


def _line_factors(t, degree):
    """1-D Lagrange factors in variable t (an affine factor), elements.py:214-219,325-335."""
    one_minus = _scale(t, -1.0, 1.0)
    if degree == 1:
        return [(1.0, [one_minus]), (1.0, [t])]
    if degree == 2:
        return [
            (1.0, [one_minus, _scale(t, -2.0, 1.0)]),
            (1.0, [t, _scale(t, 2.0, -1.0)]),
            (4.0, [t, one_minus]),
        ]
    return [
        (-0.5, [_scale(t, 1.0, -1.0), _scale(t, 3.0, -1.0), _scale(t, 3.0, -2.0)]),
        (0.5, [t, _scale(t, 3.0, -1.0), _scale(t, 3.0, -2.0)]),
        (4.5, [t, one_minus, _scale(t, -3.0, 2.0)]),
        (4.5, [t, one_minus, _scale(t, 3.0, -1.0)]),
    ]


def _simplex_factors(lams, degree):
    """Barycentric Lagrange factors; ordering of elements.py:222-231,338-358 (triangle)
    and :133-134,250-259,406-436 (tetrahedron)."""
    n = len(lams)
    out = []
    if degree == 1:
        return [(1.0, [l]) for l in lams]
    if degree == 2:
        out = [(1.0, [l, _scale(l, 2.0, -1.0)]) for l in lams]
        if n == 3:
            pairs = [(0, 1), (1, 2), (2, 0)]
        else:
            pairs = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
        out += [(4.0, [lams[a], lams[b]]) for a, b in pairs]
        return out
    out = [(0.5, [l, _scale(l, 3.0, -1.0), _scale(l, 3.0, -2.0)]) for l in lams]
    if n == 3:
        # edge 0-1: (l0-side, l1-side); 1-2; 2-0 with (l2-side first, then l0-side)
        edges = [(0, 1, 0), (0, 1, 1), (1, 2, 1), (1, 2, 2), (0, 2, 2), (0, 2, 0)]
        out += [(4.5, [lams[a], lams[b], _scale(lams[c], 3.0, -1.0)]) for a, b, c in edges]
        out.append((27.0, [lams[0], lams[1], lams[2]]))
        return out
    edges = []
    for a, b in [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]:
        edges += [(a, b, a), (a, b, b)]
    out += [(4.5, [lams[a], lams[b], _scale(lams[c], 3.0, -1.0)]) for a, b, c in edges]
    for a, b, c in [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]:
        out.append((27.0, [lams[a], lams[b], lams[c]]))
    return out


def _basis_terms(element_type, degree):
    if element_type == "tetra":
        lams = [(1.0, -1.0, -1.0, -1.0), _X, _Y, _Z]
        return _simplex_factors(lams, degree)
    if element_type == "wedge":
        tri = _simplex_factors([(1.0, -1.0, -1.0, 0.0), _X, _Y], degree)
        line = _line_factors(_Z, degree)
        return [(ct * cl, ft + fl) for cl, fl in line for ct, ft in tri]
    if element_type == "hexahedron":
        lx, ly, lz = (_line_factors(v, degree) for v in (_X, _Y, _Z))
        if degree == 1:
            corners = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0),
                       (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
            return [(lx[i][0] * ly[j][0] * lz[k][0], lx[i][1] + ly[j][1] + lz[k][1])
                    for i, j, k in corners]
        return [(lx[i][0] * ly[j][0] * lz[k][0], lx[i][1] + ly[j][1] + lz[k][1])
                for k in range(degree + 1) for j in range(degree + 1) for i in range(degree + 1)]
    raise ValueError(element_type)


def basis(element_type, degree, points):
    points = np.asarray(points, dtype=np.float64)
    flat = points.reshape(-1, 3)
    homog = np.concatenate([np.ones((len(flat), 1)), flat], axis=1)
    terms = _basis_terms(element_type, degree)
    out = np.empty((len(flat), len(terms)))
    for j, (coef, factors) in enumerate(terms):
        value = np.full(len(flat), coef)
        for f in factors:
            value = value * (homog @ np.asarray(f))
        out[:, j] = value
    return out.reshape(points.shape[:-1] + (len(terms),))


def basis_gradients(element_type, degree, points):
    points = np.asarray(points, dtype=np.float64)
    flat = points.reshape(-1, 3)
    homog = np.concatenate([np.ones((len(flat), 1)), flat], axis=1)
    terms = _basis_terms(element_type, degree)
    out = np.zeros((len(flat), len(terms), 3))
    for j, (coef, factors) in enumerate(terms):
        values = [homog @ np.asarray(f) for f in factors]
        for k, f in enumerate(factors):
            others = np.full(len(flat), coef)
            for m, v in enumerate(values):
                if m != k:
                    others = others * v
            out[:, j, :] += others[:, None] * np.asarray(f[1:])[None, :]
    return out.reshape(points.shape[:-1] + (len(terms), 3))


def corner_nodes(element_type):
    """hybrid/elements.py:35-57."""
    if element_type == "tetra":
        return np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float)
    if element_type == "wedge":
        return np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [0, 1, 1]], float)
    return np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                     [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)


def nodes(element_type, degree):
    """Solution nodes: elements.py:35-57 (P1), :234-244 (P2), :361-403 (P3)."""
    if degree == 1:
        return corner_nodes(element_type)
    third, two_thirds = 1.0 / 3.0, 2.0 / 3.0
    if degree == 2:
        line = (0.0, 1.0, 0.5)
        tri = [(0, 0), (1, 0), (0, 1), (.5, 0), (.5, .5), (0, .5)]
        tet = [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [.5, 0, 0], [0, .5, 0], [0, 0, .5],
               [.5, .5, 0], [.5, 0, .5], [0, .5, .5]]
    else:
        line = (0.0, 1.0, third, two_thirds)
        tri = [(0, 0), (1, 0), (0, 1), (third, 0), (two_thirds, 0), (two_thirds, third),
               (third, two_thirds), (0, two_thirds), (0, third), (third, third)]
        tet = [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1],
               [third, 0, 0], [two_thirds, 0, 0], [0, third, 0], [0, two_thirds, 0],
               [0, 0, third], [0, 0, two_thirds], [two_thirds, third, 0], [third, two_thirds, 0],
               [two_thirds, 0, third], [third, 0, two_thirds], [0, two_thirds, third],
               [0, third, two_thirds],
               [third, third, 0], [third, 0, third], [0, third, third], [third, third, third]]
    if element_type == "tetra":
        return np.asarray(tet, float)
    if element_type == "wedge":
        return np.asarray([[x, y, z] for z in line for x, y in tri], float)
    return np.asarray([[x, y, z] for z in line for y in line for x in line], float)


def _gauss01(order):
    raw, raw_w = np.polynomial.legendre.leggauss(order)
    return 0.5 * (raw + 1.0), 0.5 * raw_w


def volume_quadrature(element_type, degree):
    """hybrid/elements.py:60-128."""
    if degree in (2, 3):
        order = 5 if (degree == 3 or element_type in ("tetra", "wedge")) else 3
        g, w = _gauss01(order)
        pts, wts = [], []
        if element_type == "tetra":
            for a, wa in zip(g, w):
                for b, wb in zip(g, w):
                    for c, wc in zip(g, w):
                        pts.append((a, (1 - a) * b, (1 - a) * (1 - b) * c))
                        wts.append(wa * wb * wc * (1 - a) ** 2 * (1 - b))
        elif element_type == "wedge":
            for z, wz in zip(g, w):
                for a, wa in zip(g, w):
                    for b, wb in zip(g, w):
                        pts.append((a, (1 - a) * b, z))
                        wts.append(wa * wb * wz * (1 - a))
        else:
            for z, wz in zip(g, w):
                for y, wy in zip(g, w):
                    for x, wx in zip(g, w):
                        pts.append((x, y, z))
                        wts.append(wx * wy * wz)
        return np.asarray(pts), np.asarray(wts)
    if element_type == "tetra":
        a, b = 0.5854101966249685, 0.1381966011250105
        return np.array([[b, b, b], [a, b, b], [b, a, b], [b, b, a]]), np.full(4, 1.0 / 24.0)
    lp = 0.5 * (1.0 + np.array([-1.0, 1.0]) / np.sqrt(3.0))
    lw = np.full(2, 0.5)
    pts, wts = [], []
    if element_type == "wedge":
        tp = np.array([[1 / 6, 1 / 6], [2 / 3, 1 / 6], [1 / 6, 2 / 3]])
        for z, wz in zip(lp, lw):
            for (x, y) in tp:
                pts.append((x, y, z))
                wts.append(wz / 6.0)
    else:
        for z, wz in zip(lp, lw):
            for y, wy in zip(lp, lw):
                for x, wx in zip(lp, lw):
                    pts.append((x, y, z))
                    wts.append(wx * wy * wz)
    return np.asarray(pts), np.asarray(wts)


def face_quadrature(face_type, degree):
    """Face shape values (Nfq, 3|4) and weights normalised to sum 1; geometry.py:48-89."""
    if face_type == "triangle" and degree == 1:
        s = np.array([[2 / 3, 1 / 6, 1 / 6], [1 / 6, 2 / 3, 1 / 6], [1 / 6, 1 / 6, 2 / 3]])
        return s, np.full(3, 1.0 / 3.0)
    if face_type == "triangle":
        g, w = _gauss01(4 if degree <= 2 else 5)
        shapes, weights = [], []
        for a, wa in zip(g, w):
            for b, wb in zip(g, w):
                x, y = a, (1 - a) * b
                shapes.append([1 - x - y, x, y])
                weights.append(2 * wa * wb * (1 - a))
        return np.asarray(shapes), np.asarray(weights)
    g, w = _gauss01(2 if degree == 1 else (3 if degree == 2 else 4))
    shapes, weights = [], []
    for v, wv in zip(g, w):
        for u, wu in zip(g, w):
            shapes.append([(1 - u) * (1 - v), u * (1 - v), u * v, (1 - u) * v])
            weights.append(wu * wv)
    return np.asarray(shapes), np.asarray(weights)


class RefElement:
    """Per-(type, degree) tables: nodes, volume points/weights, basis at points, mass."""

    def __init__(self, element_type, degree):
        if degree not in (1, 2, 3):
            raise ValueError("Only P1, P2, and P3 are currently implemented")
        self.element_type = element_type
        self.degree = degree
        self.nodes = nodes(element_type, degree)
        self.volume_points, self.volume_weights = volume_quadrature(element_type, degree)
        self.B = basis(element_type, degree, self.volume_points)
        self.dB = basis_gradients(element_type, degree, self.volume_points)
        self.mass = np.einsum("q,qi,qj->ij", self.volume_weights, self.B, self.B)

    def basis(self, points):
        return basis(self.element_type, self.degree, points)

    def basis_gradients(self, points):
        return basis_gradients(self.element_type, self.degree, points)
