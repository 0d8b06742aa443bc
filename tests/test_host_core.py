"""Host core and C ABI tests that need no GPU: library exports, FCHK loading,
prepared AO blocks against the oracle, request validation and error mapping,
Cube output format, synthetic FCHK round trip."""
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN

import kumo_b200 as K
from kumo_b200 import synth
import oracle as O

FCHKS = ["o2.fchk.gz", "h2o_b3lyp_def2tzvp.fchk.gz", "acrolein.fchk.gz"]


def test_library_exports_every_declared_symbol():
    header = open(K.HEADER_PATH).read()
    declared = set(re.findall(r"^\s*(?:int|void|long long)\s+(kumo_\w+)\s*\(", header, flags=re.M))
    assert declared == set(K.EXPORTS)
    lib = K.lib()
    for name in declared:
        assert hasattr(lib, name), name


def test_kernels_listed_for_preloading_at_load():
    # Every launch site lists its kernel while the library loads, so the
    # preload (kumo_preload_kernels, run by kumo_server_create) covers each
    # instantiation: AO builds, both contractions of each form, orbitals,
    # potential orders, isosurface.
    assert K.registered_kernels() >= 60


@pytest.mark.parametrize("name", FCHKS)
def test_molecule_matches_oracle(name):
    path = os.path.join(GOLDEN, name)
    m = K.Molecule.from_fchk(path)
    o = O.OracleMolecule.from_fchk(path)
    info = m.info()
    assert info["nbasis"] == o.n
    assert info["nalpha"] == o.nalpha and info["nbeta"] == o.nbeta
    assert info["ao_mo_eligible"] == o.eligible
    assert info["unrestricted"] == o.unrestricted
    # Prepared blocks: l, nprim, offset, count, pure and the cutoff radius,
    # bit for bit (src/basis_evaluator.cpp:177-202).
    assert m.blocks() == o.blocks()
    z, q, xyz = m.atoms()
    assert np.array_equal(xyz.ravel(), o.atom_xyz)
    assert np.array_equal(q, o.atom_charge)


def test_check_errors_match_reference_rule():
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "o2.fchk.gz"))
    o = O.OracleMolecule.from_fchk(os.path.join(GOLDEN, "o2.fchk.gz"))
    np.testing.assert_allclose(m.info()["check_errors"], o.check_errors, rtol=1e-9, atol=1e-15)


def test_synthetic_water_round_trip(tmp_path):
    mol = synth.water(0)
    path = str(tmp_path / "water.fchk")
    synth.write_fchk(mol, path)
    m = K.Molecule.from_fchk(path)
    info = m.info()
    assert info["nbasis"] == 28 and info["nalpha"] == 5 and info["ao_mo_eligible"]
    assert info["check_errors"][1] < 1e-14
    rec = synth.read_fchk(path)
    m2 = K.Molecule.from_records(rec)
    assert m2.blocks() == m.blocks()
    o = O.OracleMolecule(rec)
    assert m.blocks() == o.blocks()


def _expect(status_cls, fn):
    with pytest.raises(status_cls) as e:
        fn()
    return str(e.value)


def test_request_validation_errors():
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "o2.fchk.gz"))
    ev = K.Evaluator(m)
    g = m.grid_around(1.0, 0.5)
    P = K.PropertyKind
    D = K.DensityComponent
    msg = _expect(K.InvalidArgument, lambda: ev.evaluate_grid(g, [K.density(P.Elf, D.Difference)]))
    assert "spin-difference" in msg
    msg = _expect(K.InvalidArgument, lambda: ev.evaluate_grid(g, [K.density(P.ReducedGradient, D.Alpha)]))
    assert "only for the total density" in msg
    msg = _expect(K.InvalidArgument, lambda: ev.evaluate_grid(g, [K.orbital(0)]))
    assert "one-based" in msg
    msg = _expect(K.OutOfRange, lambda: ev.evaluate_grid(g, [K.orbital(10_000)]))
    assert "MO index" in msg
    msg = _expect(K.InvalidArgument, lambda: ev.evaluate_grid(g, [K.density(P.SpinPolarization, D.Total)]))
    assert "spin component" in msg
    _expect(K.InvalidArgument, lambda: K.Evaluator(m, block_size=0).evaluate_grid(g, [K.density(P.Density)]))
    _expect(K.InvalidArgument, lambda: K.Evaluator(m, threshold=-1.0).evaluate_grid(g, [K.density(P.Density)]))
    _expect(K.InvalidArgument, lambda: K.Evaluator(m, block_size=70000).evaluate_grid(g, [K.density(P.Density)]))
    bad = K.Grid(np.zeros(3), np.eye(3), (0, 2, 2))
    _expect(K.InvalidArgument, lambda: ev.evaluate_grid(bad, [K.density(P.Density)]))
    dep = K.Grid(np.zeros(3), np.array([[1.0, 1.0, 0.0], [0.0, 0.0, 0.0], [0.0, 0.0, 1.0]]), (2, 2, 2))
    _expect(K.InvalidArgument, lambda: ev.evaluate_grid(dep, [K.density(P.Density)]))
    _expect(K.InvalidArgument, lambda: ev.evaluate_points(np.array([[np.nan, 0, 0]]), [K.density(P.Density)]))


def test_orbital_energy_validation_errors():
    # The checks of src/orbital_energy_fields.hpp:114-143 with their messages,
    # naming the most restrictive group requested (src/evaluator.cpp:583-588).
    P = K.PropertyKind
    D = K.DensityComponent
    o2 = K.Molecule.from_fchk(os.path.join(GOLDEN, "o2.fchk.gz"))
    g = o2.grid_around(1.0, 0.5)
    msg = _expect(K.InvalidArgument,
                  lambda: K.Evaluator(o2).evaluate_grid(g, [K.density(P.AverageLocalIonizationEnergy),
                                                            K.density(P.OrbitalWeightedFukuiPlus)]))
    assert msg.startswith("the orbital-weighted Fukui function or dual descriptor is defined only for a restricted "
                          "closed-shell calculation"), msg
    msg = _expect(K.InvalidArgument, lambda: K.Evaluator(o2).evaluate_grid(g, [K.density(P.Elf),
                                                                               K.density(P.LocalHardness, D.Alpha)]))
    assert "only for the total density" in msg
    msg = _expect(K.InvalidArgument, lambda: K.Evaluator(o2, fukui_delta=0.0).evaluate_grid(
        g, [K.density(P.OrbitalWeightedFukuiMinus)]))
    assert "fukui_delta" in msg
    rec = dict(synth.read_fchk(os.path.join(GOLDEN, "acrolein.fchk.gz")))
    # Molecule.from_records carries no orbital energies.
    m = K.Molecule.from_records(rec)
    msg = _expect(K.InvalidArgument, lambda: K.Evaluator(m).evaluate_grid(
        m.grid_around(1.0, 0.5), [K.density(P.LocalElectronAffinity)]))
    assert msg == "the local electron affinity and related fields needs the FCHK orbital energies", msg
    rec["Total SCF Density"] = np.asarray(rec["Total SCF Density"]) * 1.01
    m = K.Molecule.from_records(rec)
    msg = _expect(K.InvalidArgument, lambda: K.Evaluator(m).evaluate_grid(
        m.grid_around(1.0, 0.5), [K.density(P.AverageLocalIonizationEnergy)]))
    assert msg.startswith("the average local ionization energy needs occupied MOs that reproduce"), msg


def test_ao_mo_requires_eligible(tmp_path):
    # A density matrix that the MOs do not reproduce makes AO-MO ineligible.
    rec = synth.read_fchk(os.path.join(GOLDEN, "o2.fchk.gz"))
    rec = dict(rec)
    rec["Total SCF Density"] = np.asarray(rec["Total SCF Density"]) * 1.01
    m = K.Molecule.from_records(rec)
    assert not m.info()["ao_mo_eligible"]
    g = m.grid_around(1.0, 0.5)
    msg = _expect(K.InvalidArgument,
                  lambda: K.Evaluator(m, backend=K.Backend.AO_MO).evaluate_grid(g, [K.density(K.PropertyKind.Density)]))
    assert "not eligible" in msg


def test_fchk_errors(tmp_path):
    src = open(os.path.join(GOLDEN, "..", "..", "tests", "golden", "o2.fchk.gz"), "rb").read()
    import gzip
    text = gzip.decompress(src).decode()
    bad = tmp_path / "trunc.fchk"
    bad.write_text(text[: len(text) // 2])
    with pytest.raises(K.KumoError) as e:
        K.Molecule.from_fchk(str(bad))
    assert e.value.status == 3
    missing = tmp_path / "missing.fchk"
    missing.write_text("\n".join(l for l in text.split("\n") if not l.startswith("Shell types")))
    with pytest.raises(K.KumoError) as e:
        K.Molecule.from_fchk(str(missing))
    assert e.value.status == 3
    with pytest.raises(K.KumoError):
        K.Molecule.from_fchk(str(tmp_path / "nope.fchk"))


def test_cube_writer_layout(tmp_path):
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "o2.fchk.gz"))
    g = K.Grid(np.array([-1.0, -2.0, 0.5]), np.eye(3) * 0.25, (2, 3, 7))
    vals = np.linspace(-1e-3, 5.0, g.npoints)
    z, q, xyz = m.atoms()
    path = str(tmp_path / "f.cube")
    K.write_cube(path, g, z, q, xyz, vals, "Electron density")
    lines = open(path).read().split("\n")
    assert lines[0].startswith("chem-kumo ")
    assert lines[1] == "Electron density"
    assert lines[2] == "%5d%13.6f%13.6f%13.6f" % (2, -1.0, -2.0, 0.5)
    assert lines[3] == "%5d%13.6f%13.6f%13.6f" % (2, 0.25, 0.0, 0.0)
    # Values: %13.5e, six per line and a break after every run of 7 along k.
    body = lines[3 + 3 + 2:]
    expect = []
    row = ""
    for i, v in enumerate(vals):
        row += "%13.5e" % v
        if (i + 1) % 6 == 0 or (i + 1) % 7 == 0:
            expect.append(row)
            row = ""
    assert body[: len(expect)] == expect
    K.write_cube(str(tmp_path / "o.cube"), g, z, q, xyz, vals, "MO", orbital_index=9)
    ol = open(str(tmp_path / "o.cube")).read().split("\n")
    assert ol[2].startswith("   -2") and ol[8] == "%5d%5d" % (1, 9)
    with pytest.raises(K.InvalidArgument):
        K.write_cube(str(tmp_path / "n.cube"), g, z, q, xyz, np.full(g.npoints, np.nan))


def test_grid_around_matches_reference_formula():
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    _, _, xyz = m.atoms()
    g = m.grid_around(3.0, 0.3)
    lo, hi = xyz.min(0), xyz.max(0)
    np.testing.assert_array_equal(g.origin, lo - 3.0)
    for k in range(3):
        assert g.counts[k] == max(2, int(np.ceil((hi[k] - lo[k] + 6.0) / 0.3) + 1))


def test_cube_values_match_printf_formatting(tmp_path):
    # The threaded writer formats with to_chars; its text must equal printf's
    # %13.5e (chem-kumo's src/cube.cpp:100-110) for any double, line breaks
    # after every sixth value and after each run along the third axis.
    rng = np.random.default_rng(3)
    g = K.Grid(np.zeros(3), np.eye(3) * 0.3, (7, 5, 11))
    v = rng.standard_normal(g.npoints) * 10.0 ** rng.integers(-300, 300, g.npoints)
    v[:4] = [0.0, -0.0, 1.0, 9.999995e-5]
    path = str(tmp_path / "f.cube")
    K.write_cube(path, g, np.array([1], dtype=np.int32), np.ones(1), np.zeros((1, 3)), v)
    body = open(path).read().split("\n")[7:]
    expect, line = [], ""
    for i, x in enumerate(v):
        line += "%13.5e" % x
        if (i + 1) % 6 == 0 or (i + 1) % 11 == 0:
            expect.append(line)
            line = ""
    assert body[:len(expect)] == expect


def _o2_text():
    import gzip
    return gzip.decompress(open(os.path.join(GOLDEN, "o2.fchk.gz"), "rb").read()).decode()


def _load_text(tmp_path, text, name="t.fchk"):
    p = tmp_path / name
    p.write_text(text)
    return K.Molecule.from_fchk(str(p))


def test_fchk_record_rules(tmp_path):
    # Rules of chem-kumo's FormattedCheckpoint (src/fchk.cpp:111-186) that the
    # reader must keep: Fortran D exponents read as E, an identical duplicate
    # record is accepted, a conflicting one is rejected, values after the last
    # array value on its line are rejected, a short array is "truncated", and
    # an N=0 array takes the whole next line as its final line.
    text = _o2_text()
    base = _load_text(tmp_path, text, "base.fchk")
    ref_blocks = base.blocks()
    lines = text.split("\n")
    i = next(k for k, l in enumerate(lines) if l.startswith("Primitive exponents"))
    j = next(k for k in range(i + 1, len(lines)) if lines[k][:1].isalpha())
    d_lines = lines[:i + 1] + [l.replace("E", "D") for l in lines[i + 1:j]] + lines[j:]
    assert _load_text(tmp_path, "\n".join(d_lines), "d.fchk").blocks() == ref_blocks
    dup = lines[:j] + lines[i:j] + lines[j:]
    assert _load_text(tmp_path, "\n".join(dup), "dup.fchk").blocks() == ref_blocks
    conflict = lines[:j] + [lines[i]] + [lines[i + 1].replace("E+", "E-", 1)] + lines[i + 2:j] + lines[j:]
    with pytest.raises(K.KumoError, match="conflicting duplicate fchk record: Primitive exponents"):
        _load_text(tmp_path, "\n".join(conflict), "conflict.fchk")
    extra = list(lines)
    extra[j - 1] = extra[j - 1] + "  1.0E+00"
    with pytest.raises(K.KumoError, match="too many values on final array line in fchk: Primitive exponents"):
        _load_text(tmp_path, "\n".join(extra), "extra.fchk")
    short = list(lines)
    n = int(lines[i].split()[-1])
    short[i] = lines[i].replace(str(n), str(n + 1000))
    with pytest.raises(K.KumoError, match="invalid real token|truncated array"):
        _load_text(tmp_path, "\n".join(short), "short.fchk")
    empty_then_header = lines[:2] + ["%-43sI   N=           0" % "Empty array"] + lines[2:]
    with pytest.raises(K.KumoError, match="too many values on final array line in fchk: Empty array"):
        _load_text(tmp_path, "\n".join(empty_then_header), "empty.fchk")
    empty_then_blank = lines[:2] + ["%-43sI   N=           0" % "Empty array", ""] + lines[2:]
    assert _load_text(tmp_path, "\n".join(empty_then_blank), "empty2.fchk").blocks() == ref_blocks
    with pytest.raises(K.KumoError, match="missing its two-line header"):
        _load_text(tmp_path, "only one line", "hdr.fchk")
