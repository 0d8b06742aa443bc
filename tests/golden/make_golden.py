"""Build the golden fixtures of this directory from chem-kumo's own test data.

Run once in a checkout that has the chem-kumo sources (argument: their root):

    python tests/golden/make_golden.py /path/to/chem-kumo

It copies the three small FCHK inputs of the reference tests (O2, water
def2-TZVP, acrolein) and stores, for each reference Cube file used below, the
Cube header (origin, step vectors, counts, atoms) and a seeded sample of its
grid points with their values:

* Gaussian ``cubegen`` densities of O2 (total, alpha, beta, spin) and acrolein,
  checked in chem-kumo by ``tests/cube_reference_test.cpp:146-160``
  (max abs <= 2e-3, relative L1 <= 1e-5); Gaussian MO cubes checked by
  ``tests/orbital_reference_test.cpp`` (<= 2e-4);
* Multiwfn Cube files of derived fields of water and O2, checked by
  ``tests/multiwfn_reference_test.cpp:351-420`` (2e-5 relative, field-specific
  extras).

Gaussian Cube headers round the step to six decimals; the standard 1/6 bohr
step is restored exactly as ``tests/cube_reference_test.cpp:27-37`` does.
"""
from __future__ import annotations

import gzip
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

GAUSSIAN = [
    ("o2_density", "o2.fchk.gz", "data/o2_density.cube"),
    ("o2_alpha", "o2.fchk.gz", "data/o2_alpha.cube"),
    ("o2_beta", "o2.fchk.gz", "data/o2_beta.cube"),
    ("o2_spin", "o2.fchk.gz", "data/o2_spin.cube"),
    ("acrolein_density", "acrolein.fchk.gz", "data/acrolein_density.cube"),
    ("o2_alpha_mo_9", "o2.fchk.gz", "data/mo_reference_cubes/o2_alpha_mo_9.cube"),
    ("o2_beta_mo_7", "o2.fchk.gz", "data/mo_reference_cubes/o2_beta_mo_7.cube"),
    ("acrolein_mo_15", "acrolein.fchk.gz", "data/mo_reference_cubes/acrolein_mo_15.cube"),
]

MULTIWFN = [
    ("h2o_elf", "h2o_b3lyp_def2tzvp.fchk.gz"),
    ("h2o_rdg", "h2o_b3lyp_def2tzvp.fchk.gz"),
    ("h2o_sign_lambda2_rho", "h2o_b3lyp_def2tzvp.fchk.gz"),
    ("h2o_esp", "h2o_b3lyp_def2tzvp.fchk.gz"),
    ("h2o_lol", "h2o_b3lyp_def2tzvp.fchk.gz"),
    ("h2o_iri", "h2o_b3lyp_def2tzvp.fchk.gz"),
    ("h2o_dori", "h2o_b3lyp_def2tzvp.fchk.gz"),
    ("h2o_kinetic_k", "h2o_b3lyp_def2tzvp.fchk.gz"),
    ("h2o_kinetic_g", "h2o_b3lyp_def2tzvp.fchk.gz"),
    ("h2o_potential_energy", "h2o_b3lyp_def2tzvp.fchk.gz"),
    ("h2o_energy_density", "h2o_b3lyp_def2tzvp.fchk.gz"),
    ("h2o_shannon", "h2o_b3lyp_def2tzvp.fchk.gz"),
    ("h2o_fisher", "h2o_b3lyp_def2tzvp.fchk.gz"),
    ("h2o_elf_ts", "h2o_b3lyp_def2tzvp.fchk.gz"),
    ("h2o_lol_ts", "h2o_b3lyp_def2tzvp.fchk.gz"),
    ("o2_elf", "o2.fchk.gz"),
    ("o2_esp", "o2.fchk.gz"),
    ("o2_lol", "o2.fchk.gz"),
    ("o2_spin_polarization", "o2.fchk.gz"),
    # Orbital-energy fields (tests/REFERENCE_CUBES.md, "Orbital-energy fields"
    # and "Orbital-weighted Fukui functions").
    ("acrolein_alie", "acrolein.fchk.gz"),
    ("acrolein_lea", "acrolein.fchk.gz"),
    ("acrolein_leae", "acrolein.fchk.gz"),
    ("acrolein_local_electronegativity", "acrolein.fchk.gz"),
    ("acrolein_local_hardness", "acrolein.fchk.gz"),
    ("o2_alie", "o2.fchk.gz"),
    ("o2_lea", "o2.fchk.gz"),
    ("o2_leae", "o2.fchk.gz"),
    ("acrolein_ow_fukui_plus", "acrolein.fchk.gz"),
    ("acrolein_ow_fukui_minus", "acrolein.fchk.gz"),
    ("acrolein_ow_fukui_zero", "acrolein.fchk.gz"),
    ("acrolein_ow_dual_descriptor", "acrolein.fchk.gz"),
    ("h2o_ow_fukui_plus", "h2o_b3lyp_def2tzvp.fchk.gz"),
    ("h2o_ow_fukui_minus", "h2o_b3lyp_def2tzvp.fchk.gz"),
]

FCHK_SOURCES = {
    "o2.fchk.gz": "data/o2.fchk.gz",
    "acrolein.fchk.gz": "data/acrolein.fchk.gz",
    "h2o_b3lyp_def2tzvp.fchk.gz": "data/hybrids/h2o_b3lyp_def2tzvp.fchk.gz",
}


def read_cube(path: str):
    opener = gzip.open if path.endswith(".gz") else open
    with opener(path, "rt") as f:
        lines = f.read().split("\n")
    head = lines[2].split()
    natoms = int(head[0])
    origin = np.array([float(x) for x in head[1:4]])
    counts = []
    steps = np.zeros((3, 3))  # column a = step vector of axis a
    for a in range(3):
        parts = lines[3 + a].split()
        counts.append(int(parts[0]))
        steps[:, a] = [float(x) for x in parts[1:4]]
    atoms = []
    for i in range(abs(natoms)):
        parts = lines[6 + i].split()
        atoms.append([float(x) for x in parts[:5]])
    start = 6 + abs(natoms)
    if natoms < 0:
        start += 1  # orbital cube: "NMO index" line
    values = np.array([float(t.replace("D", "E")) for line in lines[start:] for t in line.split()])
    assert values.size == counts[0] * counts[1] * counts[2], path
    return origin, steps, np.array(counts), np.array(atoms), values


def recover_standard_step(steps: np.ndarray) -> np.ndarray:
    steps = steps.copy()
    h = 1.0 / 6.0
    for a in range(3):
        if abs(steps[a, a] - h) < 0.5e-6 + 1e-12:
            steps[a, a] = h
    return steps


def sample(values: np.ndarray, rng: np.random.Generator, n_random: int, n_top: int) -> np.ndarray:
    idx = rng.choice(values.size, size=min(n_random, values.size), replace=False)
    top = np.argsort(-np.abs(values))[:n_top]
    return np.unique(np.concatenate([idx, top]))


# Multiwfn's quantitative surface analyses (tests/multiwfn_surface_reference_test.cpp,
# run as listed in meson.build:746-785): fchk, mode, whether local extrema are compared.
SURFACES = [
    ("h2o_esp", "h2o_b3lyp_def2tzvp.fchk.gz", "esp", True),
    ("o2_esp", "o2.fchk.gz", "esp", False),
    ("acrolein_esp", "acrolein.fchk.gz", "esp", True),
    ("h2o_alie", "h2o_b3lyp_def2tzvp.fchk.gz", "alie", True),
    ("o2_alie", "o2.fchk.gz", "alie", False),
    ("acrolein_alie", "acrolein.fchk.gz", "alie", True),
    ("acrolein_leae", "acrolein.fchk.gz", "leae", True),
    ("o2_leae", "o2.fchk.gz", "leae", False),
    ("acrolein_lea", "acrolein.fchk.gz", "lea", True),
]
BOHR_IN_ANGSTROM = 0.529177210903


def _numbers(text: str):
    out = []
    for tok in text.replace("(", " ").replace(")", " ").replace("*", " ").split():
        try:
            out.append(float(tok))
        except ValueError:
            pass
    return out


def _after(lines, label, index):
    for line in lines:
        at = line.find(label)
        if at >= 0:
            return _numbers(line[at + len(label):])[index]
    raise KeyError(label)


def _extrema(lines, kind):
    label = f"The number of surface {kind}:"
    for i, line in enumerate(lines):
        if label in line:
            count = int(_after(lines, label, 0))
            rows = []
            for row in lines[i + 2:i + 2 + count]:
                v = _numbers(row)  # #, a.u., eV, kcal/mol, x, y, z (Angstrom)
                rows.append([v[1], v[4] / BOHR_IN_ANGSTROM, v[5] / BOHR_IN_ANGSTROM, v[6] / BOHR_IN_ANGSTROM])
            return rows
    return []


def surface_summaries(tests: str) -> None:
    """The numbers the reference test compares, per summary file, in atomic
    units where Multiwfn prints them, otherwise as printed (kcal/mol, eV)."""
    import json
    out = {}
    for key, fchk, mode, extrema in SURFACES:
        with open(os.path.join(tests, "data", "multiwfn", key + "_surface.txt")) as f:
            lines = f.read().splitlines()
        v = {"volume": _after(lines, "Volume:", 0), "area": _after(lines, "Overall surface area:", 0)}
        if mode == "esp":
            v.update(positive_area=_after(lines, "Positive surface area:", 0),
                     negative_area=_after(lines, "Negative surface area:", 0),
                     nonpolar_percent=_after(lines, "Nonpolar surface area (|ESP| <= 10 kcal/mol):", 1),
                     minimum_kcal=_after(lines, "Minimal value:", 0), maximum_kcal=_after(lines, "Minimal value:", 1),
                     average=_after(lines, "Overall average value:", 0),
                     positive_average=_after(lines, "Positive average value:", 0),
                     negative_average=_after(lines, "Negative average value:", 0),
                     charge_separation_kcal=_after(lines, "Internal charge separation (Pi):", 1),
                     polarity_index_kcal=_after(lines, "Molecular polarity index (MPI):", 1),
                     total_variance_kcal2=_after(lines, "Overall variance (sigma^2_tot):", 1),
                     positive_variance_kcal2=_after(lines, "Positive variance:", 1),
                     negative_variance_kcal2=_after(lines, "Negative variance:", 1),
                     balance=_after(lines, "Balance of charges (nu):", 0))
        elif mode == "alie":
            v.update(minimum=_after(lines, "Global surface minimum:", 0),
                     maximum=_after(lines, "Global surface maximum:", 0),
                     average=_after(lines, "Average value:", 0), variance=_after(lines, "Variance:", 0))
        else:
            v.update(negative_area=_after(lines, "Negative surface area:", 0),
                     minimum_ev=_after(lines, "Minimal value:", 0), maximum_ev=_after(lines, "Minimal value:", 1),
                     average_kcal=_after(lines, "Overall average value:", 2),
                     variance_kcal2=_after(lines, "Overall variance:", 2))
        entry = {"fchk": fchk, "mode": mode, "extrema": extrema, "values": v}
        if extrema:
            entry["minima"] = _extrema(lines, "minima")
            if mode == "esp":
                entry["maxima"] = _extrema(lines, "maxima")
        out[key] = entry
    with open(os.path.join(HERE, "multiwfn_surfaces.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


def main(root: str) -> None:
    tests = os.path.join(root, "tests")
    for name, rel in FCHK_SOURCES.items():
        shutil.copyfile(os.path.join(tests, rel), os.path.join(HERE, name))
    rng = np.random.default_rng(2024)
    for key, fchk, rel in GAUSSIAN:
        origin, steps, counts, atoms, values = read_cube(os.path.join(tests, rel))
        steps = recover_standard_step(steps)
        idx = sample(values, rng, 6000, 300)
        np.savez_compressed(os.path.join(HERE, f"gaussian_{key}.npz"), fchk=fchk, origin=origin,
                            steps=steps, counts=counts, atoms=atoms, index=idx.astype(np.int64),
                            values=values[idx], total_abs=np.abs(values).sum(), npoints=values.size)
    for key, fchk in MULTIWFN:
        origin, steps, counts, atoms, values = read_cube(os.path.join(tests, "data", "multiwfn", key + ".cube.gz"))
        idx = sample(values, rng, 4000, 100)
        np.savez_compressed(os.path.join(HERE, f"multiwfn_{key}.npz"), fchk=fchk, origin=origin,
                            steps=steps, counts=counts, atoms=atoms, index=idx.astype(np.int64),
                            values=values[idx], npoints=values.size)
    surface_summaries(tests)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <chem-kumo source tree>")
    main(sys.argv[1])
