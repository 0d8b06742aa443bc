"""Cube input and full-precision output (no GPU): chem-kumo's read_cube and
write_cube(CubeData) rules (src/cube.cpp:114-251) through the C ABI.  Round
trips in bohr and angstrom, gzip input, the cubegen-format files of
Field::write_cube, Fortran exponents, and every malformed-input message."""
import gzip
import os

import numpy as np
import pytest

import kumo_b200 as K

BOHR_PER_ANGSTROM = 1.8897261246257702


def _cube(counts=(5, 4, 7), seed=0, natoms=3):
    rng = np.random.default_rng(seed)
    steps = np.diag([0.25, 0.3, 0.2]) + 0.01 * rng.standard_normal((3, 3))
    grid = K.Grid(rng.standard_normal(3), steps, counts)
    z = rng.integers(1, 10, natoms).astype(np.int32)
    v = rng.standard_normal(grid.npoints) * 10.0 ** rng.integers(-8, 3, grid.npoints)
    return K.CubeData(grid, z, z.astype(float), rng.standard_normal((natoms, 3)) * 2.0, v, "first line", "second")


def test_round_trip_bohr_13_digits(tmp_path):
    c = _cube()
    path = str(tmp_path / "a.cube")
    K.write_cube_data(path, c)
    r = K.read_cube(path)
    assert (r.first_comment, r.second_comment, r.coordinates_in_angstrom) == ("first line", "second", False)
    assert r.grid.counts == c.grid.counts
    np.testing.assert_array_equal(r.values, np.array(["%.12e" % v for v in c.values], dtype=float))
    np.testing.assert_allclose(r.grid.origin, c.grid.origin, rtol=1e-12)
    np.testing.assert_allclose(r.grid.steps, c.grid.steps, rtol=1e-12, atol=1e-15)
    np.testing.assert_array_equal(r.atomic_numbers, c.atomic_numbers)
    np.testing.assert_allclose(r.xyz, c.xyz, rtol=1e-12)
    # The text itself: the header and six values per line.
    lines = open(path).read().split("\n")
    assert lines[2].split()[0] == "3" and lines[3].split()[0] == "5"
    assert len(lines[6 + 3].split()) == 6


def test_round_trip_angstrom_and_gzip(tmp_path):
    c = _cube(seed=1)
    c.coordinates_in_angstrom = True
    path = str(tmp_path / "b.cube")
    K.write_cube_data(path, c)
    head = open(path).read().split("\n")
    assert all(int(head[3 + a].split()[0]) < 0 for a in range(3))  # angstrom: negative counts
    assert abs(float(head[3].split()[1]) * BOHR_PER_ANGSTROM - c.grid.steps[0, 0]) < 1e-12
    gz = str(tmp_path / "b.cube.gz")
    with open(path, "rb") as f, gzip.open(gz, "wb") as g:
        g.write(f.read())
    for p in (path, gz):
        r = K.read_cube(p)
        assert r.coordinates_in_angstrom
        np.testing.assert_allclose(r.grid.steps, c.grid.steps, rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(r.xyz, c.xyz, rtol=1e-12, atol=1e-14)
        np.testing.assert_array_equal(r.values, np.array(["%.12e" % v for v in c.values], dtype=float))


def test_reads_cubegen_format_and_fortran_exponents(tmp_path):
    # Field::write_cube output (six significant digits, breaks after each
    # run along the third axis), and the same samples with D exponents.
    c = _cube((6, 5, 9), seed=2)
    path = str(tmp_path / "c.cube")
    K.write_cube(path, c.grid, c.atomic_numbers, c.charges, c.xyz, c.values, "Electron density")
    r = K.read_cube(path)
    assert r.first_comment.startswith("chem-kumo ") and r.second_comment == "Electron density"
    np.testing.assert_array_equal(r.values, np.array(["%13.5e" % v for v in c.values], dtype=float))
    text = open(path).read().split("\n")
    body = [l.replace("e", "D") for l in text[6 + 3:]]
    dpath = str(tmp_path / "d.cube")
    open(dpath, "w").write("\n".join(text[:6 + 3] + body))
    np.testing.assert_array_equal(K.read_cube(dpath).values, r.values)


def test_large_cube_parsed_in_ranges(tmp_path):
    # Several megabytes of samples: parsed in parallel ranges, same values.
    c = _cube((40, 50, 60), seed=3, natoms=1)
    path = str(tmp_path / "big.cube")
    K.write_cube_data(path, c)
    assert os.path.getsize(path) > 2 << 20
    np.testing.assert_array_equal(K.read_cube(path).values, np.array(["%.12e" % v for v in c.values], dtype=float))


def _header(natoms="1", nval="", axes=("3", "3", "3"), atom="6 6.0 0.0 0.0 0.0"):
    rows = ["c1", "c2", f"{natoms} 0.0 0.0 0.0 {nval}".rstrip()]
    rows += [f"{axes[a]} " + " ".join("0.2" if k == a else "0.0" for k in range(3)) for a in range(3)]
    rows += [atom] if natoms not in ("0",) else []
    return rows


@pytest.mark.parametrize("rows,samples,message", [
    (["only one line"], None, "missing Cube comments"),
    (_header(natoms="-1"), 27, "invalid Cube atom count or unsupported orbital Cube"),
    (_header(nval="2"), 27, "only scalar Cube NVAL=1 is supported"),
    (_header(nval="1 7"), 27, "malformed Cube header"),
    (_header(axes=("3", "1", "3")), 9, "invalid Cube grid axis"),
    (_header(axes=("3", "-3", "3")), 27, "mixed Cube coordinate units"),
    (_header(atom="200 6.0 0.0 0.0 0.0"), 27, "invalid Cube atom"),
    (_header(atom="6 6.0 0.0 0.0"), 27, "invalid Cube atom record"),
    (_header()[:4], None, "truncated Cube header"),
    (_header(), 28, "extra Cube samples"),
    (_header(), 26, "truncated Cube samples"),
    (_header(), -1, "invalid Cube sample"),
])
def test_malformed_cubes(tmp_path, rows, samples, message):
    text = list(rows)
    if samples is not None:
        vals = ["1.0E-03"] * abs(samples)
        if samples < 0:
            vals = ["1.0E-03"] * 26 + ["1.0x"]
        text += [" ".join(vals[i:i + 6]) for i in range(0, len(vals), 6)]
    p = tmp_path / "bad.cube"
    p.write_text("\n".join(text) + "\n")
    with pytest.raises(K.KumoError, match=message):
        K.read_cube(str(p))


def test_nval_one_and_writer_errors(tmp_path):
    rows = _header(nval="1") + [" ".join(["2.5E-01"] * 27)]
    p = tmp_path / "n.cube"
    p.write_text("\n".join(rows) + "\n")
    r = K.read_cube(str(p))
    assert r.grid.counts == (3, 3, 3) and np.all(r.values == 0.25)
    c = _cube(seed=4)
    c.first_comment = "two\nlines"
    with pytest.raises(K.InvalidArgument, match="single lines"):
        K.write_cube_data(str(tmp_path / "x.cube"), c)
    c = _cube(seed=4)
    c.values[3] = np.nan
    with pytest.raises(K.InvalidArgument, match="nonfinite Cube sample"):
        K.write_cube_data(str(tmp_path / "x.cube"), c)
    bad = tmp_path / "bad.cube.gz"
    bad.write_bytes(gzip.compress(open(p, "rb").read())[:-6])
    with pytest.raises(K.KumoError):
        K.read_cube(str(bad))
    with pytest.raises(K.KumoError, match="cannot open"):
        K.read_cube(str(tmp_path / "missing.cube"))
