"""Molecular surfaces: the isosurface construction (marching tetrahedra on the
device, Newton placement of the vertices), surface statistics, the potential,
ionization-energy and mapped surfaces, and PLY output.

The CPU oracle (oracle/surface.py) is pinned first against the analytic
checks of tests/molecular_surface_test.cpp:56-280 (a sphere as the isosurface
of -|r|, a regular octahedron with exact statistics); the device surfaces are
then compared with it: the same vertex and triangle numbering, vertices within
1e-9 bohr.
"""
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN, scaled_error

import kumo_b200 as K
import oracle as O
import surface as OS

P = K.PropertyKind


def _closed_euler(tri: np.ndarray, nv: int) -> int:
    """Every directed edge once and its reverse once; returns V - E + F."""
    edges = {}
    for t in tri:
        for a in range(3):
            e = (int(t[a]), int(t[(a + 1) % 3]))
            edges[e] = edges.get(e, 0) + 1
    bad = sum(1 for e, c in edges.items() if c != 1 or (e[1], e[0]) not in edges)
    assert bad == 0
    return nv - len(edges) // 2 + len(tri)


def _cube_grid(half, spacing):
    origin = np.full(3, -half) + np.array([0.013, 0.007, 0.021])
    n = int(math.ceil(2 * half / spacing)) + 1
    return origin, np.eye(3) * spacing, (n, n, n)


def _sphere_inputs(radius, spacing):
    origin, steps, counts = _cube_grid(radius + 1.0, spacing)
    idx = np.indices(counts).reshape(3, -1).T
    pts = origin[None, :] + idx @ steps.T
    samples = -np.linalg.norm(pts, axis=1)

    def f(p):
        r = np.linalg.norm(p, axis=1)
        return -r, -p / r[:, None]

    return origin, steps, counts, samples, f


def _octahedron():
    v = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], dtype=float)
    tri = []
    for x in (0, 1):
        for y in (2, 3):
            for z in (4, 5):
                t = [x, y, z]
                if np.dot(np.cross(v[y] - v[x], v[z] - v[x]), v[x]) < 0:
                    t[1], t[2] = t[2], t[1]
                tri.append(t)
    return v, np.array(tri, dtype=np.int64)


# -- the oracle against analytic answers (CPU) --------------------------------
def test_oracle_sphere():
    radius = 1.7
    prev = None
    for spacing in (0.2, 0.1):
        origin, steps, counts, samples, f = _sphere_inputs(radius, spacing)
        x, tri, _ = OS.extract_isosurface(origin, steps, counts, samples, -radius, f)
        assert _closed_euler(tri, len(x)) == 2
        assert np.max(np.abs(np.linalg.norm(x, axis=1) - radius)) <= 1e-9
        a, b, c = x[tri[:, 0]], x[tri[:, 1]], x[tri[:, 2]]
        area = 0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1).sum()
        ctr = x.mean(0)
        volume = np.einsum("ij,ij->i", a - ctr, np.cross(b - ctr, c - ctr)).sum() / 6.0
        ea = (4 * math.pi * radius ** 2 - area) / (4 * math.pi * radius ** 2)
        ev = (4 / 3 * math.pi * radius ** 3 - volume) / (4 / 3 * math.pi * radius ** 3)
        assert 0 < ea < 3e-3 and 0 < ev < 6e-3
        if prev:
            assert prev[0] / ea > 3 and prev[1] / ev > 3
        prev = (ea, ev)


def test_oracle_statistics_sphere():
    radius, spacing = 1.7, 0.2
    origin, steps, counts, samples, f = _sphere_inputs(radius, spacing)
    x, tri, _ = OS.extract_isosurface(origin, steps, counts, samples, -radius, f)
    n = np.array([0.3, 0.2, 0.9])
    n /= np.linalg.norm(n)
    s = OS.statistics(x, tri, x @ n, 0.4)
    rel = 4e-3
    assert abs(s["positive_area"] / s["area"] - 0.5) <= rel
    assert abs(s["positive_average"] - radius / 2) <= rel * radius / 2
    assert abs(s["positive_variance"] - radius ** 2 / 12) <= rel * radius ** 2 / 12
    assert abs(s["balance"] - 0.25) <= 1e-6
    assert abs(s["nonpolar_area"] - 4 * math.pi * radius * 0.4) <= rel * 4 * math.pi * radius * 0.4
    assert len(s["local_minima"]) == 1 and len(s["local_maxima"]) == 1


def test_statistics_octahedron():
    # Exact answers of the linear interpolation on a regular octahedron with
    # V = x (tests/molecular_surface_test.cpp:171-280), through the C ABI.
    v, tri = _octahedron()
    x = v[:, 0].copy()
    r3 = math.sqrt(3.0)
    s = K.surface_statistics(v, tri, x, 0.5)
    t = 1e-14
    for key, want in [("area", 4 * r3), ("positive_area", 2 * r3), ("negative_area", 2 * r3),
                      ("positive_average", 1 / 3), ("negative_average", -1 / 3), ("positive_variance", 1 / 18),
                      ("negative_variance", 1 / 18), ("total_variance", 1 / 9), ("balance", 0.25),
                      ("charge_separation", 1 / 3), ("polarity_index", 1 / 3), ("nonpolar_area", 3 * r3)]:
        assert abs(s[key] - want) <= t * abs(want), key
    assert abs(s["average"]) <= t
    assert s["minimum_vertex"] == 1 and s["maximum_vertex"] == 0 and s["minimum"] == -1 and s["maximum"] == 1
    assert s["local_minima"] == [1] and s["local_maxima"] == [0]
    u = K.surface_statistics(v, tri, x + 0.25)
    assert abs(u["negative_area"] - 9 * r3 / 8) <= t * 9 * r3 / 8
    assert abs(u["average"] - 0.25) <= t and abs(u["negative_average"] + 0.25) <= t
    p = K.surface_statistics(v, tri, x + 2.0)
    assert p["negative_area"] == 0 and math.isnan(p["negative_average"]) and p["negative_variance"] == 0
    assert p["balance"] == 0
    c = K.surface_statistics(v, tri, np.full(6, 2.0))
    assert c["total_variance"] == 0 and math.isnan(c["balance"]) and c["nonpolar_area"] == 0
    assert c["local_minima"] == [] and c["local_maxima"] == []
    # The oracle gives the same numbers.
    so = OS.statistics(v, tri, x, 0.5)
    for key in ("area", "positive_area", "positive_variance", "charge_separation", "nonpolar_area"):
        assert abs(so[key] - s[key]) <= 1e-14
    with pytest.raises(K.InvalidArgument):
        K.surface_statistics(v, tri, np.zeros(5))
    with pytest.raises(K.InvalidArgument):
        K.surface_statistics(v, tri, np.where(np.arange(6) == 2, np.nan, x))
    with pytest.raises(K.InvalidArgument):
        K.surface_statistics(v, tri, x, -1.0)
    bad = tri.copy()
    bad[0, 1] = 6
    with pytest.raises(K.InvalidArgument):
        K.surface_statistics(v, bad, x)
    with pytest.raises(K.InvalidArgument):
        K.surface_statistics(np.zeros_like(v), tri, x)


def test_statistics_match_oracle_on_sphere_mesh():
    radius, spacing = 1.7, 0.2
    origin, steps, counts, samples, f = _sphere_inputs(radius, spacing)
    x, tri, _ = OS.extract_isosurface(origin, steps, counts, samples, -radius, f)
    vals = np.sin(3 * x[:, 0]) * np.cos(2 * x[:, 1]) + 0.1 * x[:, 2]
    s = K.surface_statistics(x, tri, vals, 0.3)
    so = OS.statistics(x, tri, vals, 0.3)
    for key in ("area", "positive_area", "negative_area", "nonpolar_area", "average", "positive_average",
                "negative_average", "positive_variance", "negative_variance", "balance", "charge_separation",
                "polarity_index"):
        assert abs(s[key] - so[key]) <= 1e-12 * max(1.0, abs(so[key])), key
    assert s["local_minima"] == so["local_minima"] and s["local_maxima"] == so["local_maxima"]
    assert s["minimum_vertex"] == so["minimum_vertex"] and s["maximum_vertex"] == so["maximum_vertex"]


def test_write_ply(tmp_path):
    v, tri = _octahedron()
    path = tmp_path / "o.ply"
    K.write_ply(str(path), v, tri, [("esp", v[:, 0] * 0.25)], ["made by a test"])
    lines = path.read_text().splitlines()
    assert lines[:11] == ["ply", "format ascii 1.0", "comment made by a test", "element vertex 6", "property double x",
                          "property double y", "property double z", "property double esp", "element face 8",
                          "property list uchar int vertex_indices", "end_header"]
    assert lines[11] == "1.000000000e+00 0.000000000e+00 0.000000000e+00 2.500000000e-01"
    assert lines[17] == "3 " + " ".join(str(int(i)) for i in tri[0])
    assert len(lines) == 11 + 6 + 8
    for fields, comments in [([("x", v[:, 0])], []), ([("a b", v[:, 0])], []), ([("e", v[:3, 0])], []),
                             ([("e", np.full(6, np.inf))], []), ([], ["two\nlines"]),
                             ([("e", v[:, 0]), ("e", v[:, 1])], [])]:
        with pytest.raises(K.InvalidArgument):
            K.write_ply(str(tmp_path / "bad.ply"), v, tri, fields, comments)


def test_surface_argument_errors_before_device_work():
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "o2.fchk.gz"))
    with pytest.raises(K.InvalidArgument, match="at least 1e-8"):
        K.density_isosurface(m, 1e-9)
    with pytest.raises(K.InvalidArgument, match="spacing"):
        K.density_isosurface(m, 1e-3, 0.0)
    with pytest.raises(K.InvalidArgument, match="potential tolerance"):
        K.electrostatic_potential_surface(m, potential_tolerance=-1.0)
    with pytest.raises(K.InvalidArgument, match="no property"):
        K.map_on_density_isosurface(m, [])
    with pytest.raises(K.InvalidArgument, match="one-component"):
        K.map_on_density_isosurface(m, [K.density(P.Gradient)])


# -- the device surfaces against the oracle (GPU) -----------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("spacing", [0.2, 0.1])
def test_extract_sphere_matches_oracle(spacing):
    radius = 1.7
    origin, steps, counts, samples, f = _sphere_inputs(radius, spacing)
    s = K.extract_isosurface(K.Grid(origin, steps, counts), samples, -radius, f)
    x, tri, cells = OS.extract_isosurface(origin, steps, counts, samples, -radius, f)
    assert s.vertices.shape == x.shape and np.array_equal(s.triangles, tri)
    assert np.array_equal(s.cells, cells)
    assert np.max(np.abs(s.vertices - x)) <= 1e-12
    assert _closed_euler(s.triangles, len(s.vertices)) == 2
    # Nothing above the isovalue: an empty mesh; the surface reaching the
    # boundary is an error.
    e = K.extract_isosurface(K.Grid(origin, steps, counts), samples, 1.0, f)
    assert len(e.vertices) == 0 and len(e.triangles) == 0
    with pytest.raises(K.InvalidArgument, match="boundary"):
        K.extract_isosurface(K.Grid(origin, steps, counts), samples, -100.0, f)


def _oracle_density_surface(name, isovalue, spacing):
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, name))
    o = O.OracleMolecule.from_fchk(os.path.join(GOLDEN, name))
    for margin in np.arange(4.0, 16.5, 2.0):
        g = m.grid_around(margin, spacing)
        outs, _ = o.evaluate([(0, 0, 0, 0)], grid=(g.origin, g.steps, g.counts), backend=1)
        rho = outs[0][0]
        f = rho.reshape(g.counts)
        face = np.concatenate([f[0].ravel(), f[-1].ravel(), f[:, 0].ravel(), f[:, -1].ravel(), f[:, :, 0].ravel(),
                               f[:, :, -1].ravel()])
        if np.any(face >= isovalue):
            continue

        def func(p):
            r, _ = o.evaluate([(0, 0, 0, 0), (1, 0, 0, 0)], points=p, backend=1)
            return r[0][0], r[1].T

        return m, o, OS.extract_isosurface(g.origin, g.steps, g.counts, rho, isovalue, func)
    raise AssertionError("no closed surface")


@pytest.mark.gpu
@pytest.mark.parametrize("name,spacing", [("h2o_b3lyp_def2tzvp.fchk.gz", 0.3), ("o2.fchk.gz", 0.35)])
def test_density_isosurface_matches_oracle(name, spacing):
    m, o, (x, tri, _) = _oracle_density_surface(name, 1e-3, spacing)
    s = K.density_isosurface(m, 1e-3, spacing)
    assert np.array_equal(s.triangles, tri)
    assert np.max(np.abs(s.vertices - x)) <= 1e-9
    assert _closed_euler(s.triangles, len(s.vertices)) == 2
    rho, _ = K.Evaluator(m, backend=K.Backend.AO_P).evaluate_points(s.vertices, [K.density(P.Density)])
    assert np.max(np.abs(rho[0][0] - 1e-3)) <= 1e-12


@pytest.mark.gpu
def test_potential_and_ionization_surfaces():
    name = "h2o_b3lyp_def2tzvp.fchk.gz"
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, name))
    o = O.OracleMolecule.from_fchk(os.path.join(GOLDEN, name))
    mesh = K.density_isosurface(m, 1e-3, 0.3)
    es = K.electrostatic_potential_surface(m, 1e-3, 0.3, potential_tolerance=1e-8)
    assert np.array_equal(es.vertices, mesh.vertices) and np.array_equal(es.triangles, mesh.triangles)
    ref = O.OracleESP(o).evaluate(es.vertices)
    # potential_tolerance: every value within 1e-8 of the exact potential
    # (pairs whose bounds sum to at most half of it are left out); with
    # tolerance 0 the surface values are the exact ones to rounding.
    assert np.max(np.abs(es.values[0] - ref)) <= 1e-8
    exact = K.electrostatic_potential_surface(m, 1e-3, 0.3, potential_tolerance=0.0)
    assert scaled_error(exact.values[0], ref) <= 1e-12
    st = K.surface_statistics(es.vertices, es.triangles, es.values[0])
    assert st == es.statistics[0] or all(
        (st[k] == es.statistics[0][k]) or (isinstance(st[k], float) and math.isnan(st[k]))
        for k in st)
    assert st["negative_area"] > 0 and st["positive_area"] > 0
    ie = K.local_ionization_energy_surface(m, 1e-3, 0.3)
    alie = O.orbital_energy_fields(o, ie.vertices, [19])[0]
    assert scaled_error(ie.values[0], alie) <= 1e-12
    assert ie.statistics[0]["negative_area"] == 0 and ie.statistics[0]["minimum"] > 0
    pts = np.array([[0.1, 0.2, 0.3], [1.0, -0.5, 0.2]])
    got = K.average_local_ionization_energy(m, pts)
    assert scaled_error(got, O.orbital_energy_fields(o, pts, [19])[0]) <= 1e-12


@pytest.mark.gpu
def test_map_on_density_isosurface():
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    homo = int(m.info()["nalpha"])
    props = [K.density(P.Elf), K.orbital(homo), K.density(P.Elf), K.density(P.ElectrostaticPotential)]
    s, used = K.map_on_density_isosurface(m, props, 1e-3, 0.35)
    assert len(s.values) == 3 and used == int(K.Backend.AO_MO)
    ref, _ = K.Evaluator(m).evaluate_points(s.vertices, [props[0], props[1], props[3]])
    for a, r in zip(s.values, ref):
        assert np.array_equal(a, r[0])
    assert s.statistics[0]["nonpolar_area"] == 0.0


# -- against Multiwfn's surface analyses (tests/multiwfn_surface_reference_test.cpp) --
def _surface_refs():
    import json
    with open(os.path.join(GOLDEN, "multiwfn_surfaces.json")) as f:
        return json.load(f)


KCAL, EV = 627.51, 27.2113838  # Multiwfn's conversion factors


def _close(actual, expected, rel, abs_, what):
    tol = max(abs_, rel * abs(expected))
    assert abs(actual - expected) <= tol, f"{what}: {actual} vs {expected} (tolerance {tol})"


def _extrema_match(surf, values, found, expected, tol, what):
    assert len(found) == len(expected), what
    used = set()
    for val, x, y, z in expected:
        d = [np.linalg.norm(surf.vertices[f] - np.array([x, y, z])) if i not in used else np.inf
             for i, f in enumerate(found)]
        best = int(np.argmin(d))
        used.add(best)
        assert d[best] <= 0.4, what
        _close(values[found[best]], val, 0.0, tol, what)


@pytest.mark.gpu
@pytest.mark.parametrize("key", ["h2o_esp", "o2_esp", "acrolein_esp", "h2o_alie", "o2_alie", "acrolein_alie",
                                 "acrolein_leae", "o2_leae", "acrolein_lea"])
def test_multiwfn_surface_analyses(key):
    # Multiwfn at 0.05 bohr against the default 0.25 bohr, at the reference
    # test's tolerances (about three times the differences it observed).
    ref = _surface_refs()[key]
    v = ref["values"]
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, ref["fchk"]))
    mode = ref["mode"]
    if mode == "esp":
        s = K.electrostatic_potential_surface(m)
    elif mode == "alie":
        s = K.local_ionization_energy_surface(m)
    else:
        kind = P.LocalElectronAttachmentEnergy if mode == "leae" else P.LocalElectronAffinity
        s, _ = K.map_on_density_isosurface(m, [K.density(kind)], 4e-3 if mode == "leae" else 1e-3)
    st, vals = s.statistics[0], s.values[0]
    _close(s.volume(), v["volume"], 5e-3, 0, "volume")
    _close(st["area"], v["area"], 5e-3, 0, "area")
    if mode == "esp":
        _close(st["positive_area"], v["positive_area"], 5e-3, 0, "A+")
        _close(st["negative_area"], v["negative_area"], 5e-3, 0, "A-")
        _close(st["nonpolar_area"] / st["area"], v["nonpolar_percent"] / 100, 0, 2e-3, "nonpolar fraction")
        _close(st["minimum"], v["minimum_kcal"] / KCAL, 0, 4e-5, "minimum")
        _close(st["maximum"], v["maximum_kcal"] / KCAL, 0, 4e-5, "maximum")
        for name in ("average", "positive_average", "negative_average"):
            _close(st[name], v[name], 5e-3, 2e-6, name)
        _close(st["charge_separation"], v["charge_separation_kcal"] / KCAL, 5e-3, 2e-6, "Pi")
        _close(st["polarity_index"], v["polarity_index_kcal"] / KCAL, 5e-3, 2e-6, "MPI")
        for name in ("total_variance", "positive_variance", "negative_variance"):
            _close(st[name], v[name + "_kcal2"] / KCAL ** 2, 1e-2, 2e-8, name)
        _close(st["balance"], v["balance"], 0, 1e-3, "nu")
        if ref["extrema"]:
            _extrema_match(s, vals, st["local_minima"], ref["minima"], 4e-5, "minima")
            _extrema_match(s, vals, st["local_maxima"], ref["maxima"], 4e-5, "maxima")
    elif mode == "alie":
        _close(st["positive_area"], st["area"], 1e-14, 0, "A+ = A")
        assert st["negative_area"] == 0.0
        _close(st["minimum"], v["minimum"], 0, 4e-5, "minimum")
        _close(st["maximum"], v["maximum"], 0, 4e-4, "maximum")
        _close(st["average"], v["average"], 5e-5, 0, "average")
        _close(st["total_variance"], v["variance"], 2e-2, 0, "variance")
        if ref["extrema"]:
            _extrema_match(s, vals, st["local_minima"], ref["minima"], 8e-4, "minima")
    else:
        glob, minima, avg, var = (1.5e-6, 6e-5, 1e-3, 2.5e-2) if mode == "leae" else (4e-5, 6e-3, 1.5e-4, 5e-3)
        _close(st["negative_area"], v["negative_area"], 5e-3, 0, "A-")
        _close(st["minimum"], v["minimum_ev"] / EV, 0, glob, "minimum")
        _close(st["maximum"], v["maximum_ev"] / EV, 0, glob, "maximum")
        _close(st["average"], v["average_kcal"] / KCAL, avg, 0, "average")
        _close(st["total_variance"], v["variance_kcal2"] / KCAL ** 2, var, 0, "variance")
        if ref["extrema"]:
            _extrema_match(s, vals, st["local_minima"], ref["minima"], minima, "minima")
