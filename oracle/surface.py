"""CPU restatement of chem-kumo's isosurface construction and surface
statistics (src/surface.cpp:66-531), in numpy and plain Python loops.

TEST INFRASTRUCTURE ONLY: the checker of the device surfaces.  Only tests/
import this module.
"""
from __future__ import annotations

import math
from typing import Callable, Dict, List, Sequence, Tuple

import numpy as np

# Tetrahedra around the main diagonal (src/surface.cpp:73-76).
TETRAHEDRA = ((0, 1, 3, 7), (0, 1, 5, 7), (0, 2, 3, 7), (0, 2, 6, 7), (0, 4, 5, 7), (0, 4, 6, 7))


def _offset(mask: int) -> Tuple[int, int, int]:
    return mask & 1, (mask >> 1) & 1, mask >> 2


def grid_point(origin, steps, counts, linear: int) -> np.ndarray:
    """origin + steps (i, j, k) for a Field-order index (src/grid_geometry.hpp:59-68)."""
    ny, nz = counts[1], counts[2]
    i, j, k = linear // (ny * nz), (linear // nz) % ny, linear % nz
    s = np.asarray(steps, dtype=float)
    return np.array([origin[r] + ((s[r, 0] * i + s[r, 1] * j) + s[r, 2] * k) for r in range(3)])


def _tetrahedron_polygon(masks, inside, pos):
    """src/surface.cpp:87-129."""
    ins = [m for m in masks if inside[m]]
    outs = [m for m in masks if not inside[m]]
    if not ins or not outs:
        return []
    if len(ins) == 1:
        ends = [(ins[0], outs[0]), (ins[0], outs[1]), (ins[0], outs[2])]
    elif len(outs) == 1:
        ends = [(ins[0], outs[0]), (ins[1], outs[0]), (ins[2], outs[0])]
    else:
        ends = [(ins[0], outs[0]), (ins[0], outs[1]), (ins[1], outs[1]), (ins[1], outs[0])]
    mid = [0.5 * (pos[a] + pos[b]) for a, b in ends]
    if len(ends) == 3:
        normal = np.cross(mid[1] - mid[0], mid[2] - mid[0])
    else:
        normal = np.cross(mid[2] - mid[0], mid[3] - mid[1])
    outward = sum(pos[m] / len(outs) for m in outs) - sum(pos[m] / len(ins) for m in ins)
    if float(np.dot(normal, outward)) < 0:
        ends = ends[::-1]
    return ends


def polygonize(origin, steps, counts, samples: np.ndarray, iso: float):
    """Marching tetrahedra, cells k fastest; vertices numbered at first
    appearance (src/surface.cpp:150-200).  Returns edges [(inside, outside,
    cell)] and polygons [[vertex ids]]."""
    nx, ny, nz = counts
    f = np.asarray(samples, dtype=float).reshape(nx, ny, nz)
    ins = f >= iso
    c = np.zeros((nx - 1, ny - 1, nz - 1), dtype=np.int32)
    for m in range(8):
        a, b, d = _offset(m)
        c += ins[a:a + nx - 1, b:b + ny - 1, d:d + nz - 1]
    mixed = np.argwhere((c > 0) & (c < 8))  # lexicographic (i, j, k): the sweep order
    edges: List[Tuple[int, int, Tuple[int, int, int]]] = []
    polygons: List[List[int]] = []
    ids: Dict[Tuple[int, int], int] = {}
    for i, j, k in mixed:
        corner = [((i + a) * ny + (j + b)) * nz + (k + d) for a, b, d in map(_offset, range(8))]
        inside = [bool(f.flat[q] >= iso) for q in corner]
        pos = [grid_point(origin, steps, counts, q) for q in corner]
        for tet in TETRAHEDRA:
            ends = _tetrahedron_polygon(tet, inside, pos)
            if not ends:
                continue
            poly = []
            for a, b in ends:
                low, high = min(a, b), max(a, b)
                key = (corner[low], high ^ low)
                if key not in ids:
                    ids[key] = len(edges)
                    oa, ob, od = _offset(low)
                    edges.append((corner[a], corner[b], (int(i + oa), int(j + ob), int(k + od))))
                poly.append(ids[key])
            polygons.append(poly)
    return edges, polygons


def place_vertices(origin, steps, counts, samples, iso, edges, function: Callable, tolerance=1e-10,
                   max_iterations=200) -> np.ndarray:
    """Safeguarded Newton steps along each edge (src/surface.cpp:203-259);
    function(points (n, 3)) -> (values, gradients (n, 3))."""
    f = np.asarray(samples, dtype=float).ravel()
    n = len(edges)
    a = np.array([grid_point(origin, steps, counts, e[0]) for e in edges]).reshape(n, 3)
    b = np.array([grid_point(origin, steps, counts, e[1]) for e in edges]).reshape(n, 3)
    fa = np.array([f[e[0]] for e in edges])
    fb = np.array([f[e[1]] for e in edges])
    t = np.clip((fa - iso) / (fa - fb), 0.0, 1.0) if n else np.zeros(0)
    low, high = np.zeros(n), np.ones(n)
    active = list(range(n))
    it = 0
    while active:
        if it == max_iterations:
            raise RuntimeError("isosurface vertices did not converge")
        it += 1
        idx = np.array(active)
        d = b[idx] - a[idx]
        pts = a[idx] + t[idx][:, None] * d
        vals, grads = function(pts)
        nxt = []
        for p, v in enumerate(active):
            g = vals[p] - iso
            if g == 0.0:
                continue
            if g > 0.0:
                low[v] = t[v]
            else:
                high[v] = t[v]
            length = math.sqrt(float(d[p] @ d[p]))
            step = t[v] - g / float(grads[p] @ d[p])
            if not (low[v] < step < high[v]):
                step = 0.5 * (low[v] + high[v])
            moved = abs(step - t[v]) * length
            t[v] = step
            if moved > tolerance and (high[v] - low[v]) * length > tolerance:
                nxt.append(v)
        active = nxt
    return a + t[:, None] * (b - a) if n else np.zeros((0, 3))


def triangulate(polygons, x: np.ndarray) -> np.ndarray:
    """src/surface.cpp:262-281."""
    tri = []
    for p in polygons:
        if len(p) == 3:
            tri.append(p)
        elif np.sum((x[p[0]] - x[p[2]]) ** 2) <= np.sum((x[p[1]] - x[p[3]]) ** 2):
            tri += [[p[0], p[1], p[2]], [p[0], p[2], p[3]]]
        else:
            tri += [[p[0], p[1], p[3]], [p[1], p[2], p[3]]]
    return np.array(tri, dtype=np.int64).reshape(-1, 3)


def extract_isosurface(origin, steps, counts, samples, iso, function):
    edges, polys = polygonize(origin, steps, counts, samples, iso)
    x = place_vertices(origin, steps, counts, samples, iso, edges, function)
    cells = np.array([e[2] for e in edges], dtype=np.int64).reshape(-1, 3)
    return x, triangulate(polys, x), cells


# -- statistics (src/surface.cpp:355-531) -------------------------------------
def _clip(x, v, level, upper):
    keep = (lambda w: w >= level) if upper else (lambda w: w < level)
    px, pv = [], []
    for i in range(3):
        j = (i + 1) % 3
        ki, kj = keep(v[i]), keep(v[j])
        if ki:
            px.append(x[i])
            pv.append(v[i])
        if ki != kj:
            s = (level - v[i]) / (v[j] - v[i])
            px.append(x[i] + s * (x[j] - x[i]))
            pv.append(level)
    out = []
    for i in range(1, len(px) - 1):
        out.append((0.5 * np.linalg.norm(np.cross(px[i] - px[0], px[i + 1] - px[0])), pv[0], pv[i], pv[i + 1]))
    return out


def _sq(area, w0, w1, w2, s):
    a, b, c = w0 - s, w1 - s, w2 - s
    return area / 6.0 * (a * a + b * b + c * c + a * b + b * c + c * a)


def statistics(vertices: np.ndarray, triangles: np.ndarray, values: Sequence[float],
               polar_threshold: float = 10.0 / 627.5094740631) -> Dict[str, object]:
    x = np.asarray(vertices, dtype=float)
    v = np.asarray(values, dtype=float)
    s = dict(positive_area=0.0, negative_area=0.0)
    pi = ni = above = below = 0.0
    for t in triangles:
        xs, vs = x[list(t)], v[list(t)]
        for a, w0, w1, w2 in _clip(xs, vs, 0.0, True):
            s["positive_area"] += a
            pi += a * (w0 + w1 + w2) / 3.0
        for a, w0, w1, w2 in _clip(xs, vs, 0.0, False):
            s["negative_area"] += a
            ni += a * (w0 + w1 + w2) / 3.0
        above += sum(p[0] for p in _clip(xs, vs, polar_threshold, True))
        below += sum(p[0] for p in _clip(xs, vs, -polar_threshold, False))
    area = s["positive_area"] + s["negative_area"]
    s["area"] = area
    s["average"] = (pi + ni) / area
    s["positive_average"] = pi / s["positive_area"] if s["positive_area"] > 0 else math.nan
    s["negative_average"] = ni / s["negative_area"] if s["negative_area"] > 0 else math.nan
    s["polarity_index"] = (pi - ni) / area
    s["nonpolar_area"] = max(0.0, area - above - below)
    ps = ns = dev = 0.0
    for t in triangles:
        xs, vs = x[list(t)], v[list(t)]
        if s["positive_area"] > 0:
            ps += sum(_sq(*p, s["positive_average"]) for p in _clip(xs, vs, 0.0, True))
        if s["negative_area"] > 0:
            ns += sum(_sq(*p, s["negative_average"]) for p in _clip(xs, vs, 0.0, False))
        dev += sum(a * ((w0 + w1 + w2) / 3.0 - s["average"]) for a, w0, w1, w2 in _clip(xs, vs, s["average"], True))
        dev += sum(a * (s["average"] - (w0 + w1 + w2) / 3.0) for a, w0, w1, w2 in _clip(xs, vs, s["average"], False))
    s["positive_variance"] = ps / s["positive_area"] if s["positive_area"] > 0 else 0.0
    s["negative_variance"] = ns / s["negative_area"] if s["negative_area"] > 0 else 0.0
    tv = s["positive_variance"] + s["negative_variance"]
    s["total_variance"] = tv
    s["balance"] = s["positive_variance"] * s["negative_variance"] / (tv * tv) if tv > 0 else math.nan
    s["charge_separation"] = dev / area
    s["minimum_vertex"] = int(np.argmin(v))
    s["maximum_vertex"] = int(np.argmax(v))
    s["minimum"], s["maximum"] = float(v.min()), float(v.max())
    nb = [set() for _ in range(len(v))]
    for t in triangles:
        for a in range(3):
            nb[t[a]].update((t[(a + 1) % 3], t[(a + 2) % 3]))

    def extremum(i, beyond):
        if not nb[i]:
            return False
        for j in nb[i]:
            if j == i:
                continue
            if not beyond(v[i], v[j]):
                return False
            if any(k != i and not beyond(v[i], v[k]) for k in nb[j]):
                return False
        return True

    mins = [i for i in range(len(v)) if extremum(i, lambda p, q: p < q)]
    maxs = [i for i in range(len(v)) if extremum(i, lambda p, q: p > q)]
    s["local_minima"] = sorted(mins, key=lambda i: (v[i], i))
    s["local_maxima"] = sorted(maxs, key=lambda i: (-v[i], i))
    return s
