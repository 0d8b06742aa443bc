"""Seeded synthetic molecules written as Gaussian formatted checkpoint (FCHK) files.

The benchmark workloads are synthetic molecules with random contracted Gaussian
bases, a random S-orthonormal orbital matrix C and the density matrices built
from it, written in the FCHK text format that chem-kumo reads
(``src/fchk.cpp:78-187``, ``src/basis.cpp:21-120``, ``src/molecule.cpp:20-180``),
so that the reference and this library read identical bytes.

Conventions followed (reference files cited for each):

* Gaussian Cartesian component order, ``src/basis_evaluator.cpp:135-152``.
* Primitive normalisation ``(2a/pi)^(3/4) sqrt((4a)^l / prod (2n-1)!!)``,
  ``src/basis_math.cpp:17-25``; the reference multiplies the file's contraction
  coefficients by this factor only (``src/basis_math.cpp:41-45``), so the
  generator normalises each contracted function itself.
* Pure (spherical) shells use the Schlegel-Frisch Cartesian-to-pure map in
  Gaussian m order 0, +1, -1, ... (``src/basis_evaluator.cpp:49-83,157-175``).
* Packed lower-triangle density matrices, row-major with i >= j
  (``src/molecule.cpp:20-33``); MO coefficients MO by MO, AO fastest
  (``src/mo_coefficients.hpp:21-34``).

The overlap matrix needed for the S-orthonormal orbitals is computed here with
an Obara-Saika recursion over primitive pairs (vectorised with numpy).
"""
from __future__ import annotations

import gzip
import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

ELEMENT_Z = {"H": 1, "C": 6, "N": 7, "O": 8}

# ---------------------------------------------------------------------------
# Angular helpers
# ---------------------------------------------------------------------------


def cartesian_order(l: int) -> List[Tuple[int, int, int]]:
    """Gaussian FCHK order of the Cartesian components of a shell of momentum l."""
    if l == 0:
        return [(0, 0, 0)]
    if l == 1:
        return [(1, 0, 0), (0, 1, 0), (0, 0, 1)]
    if l == 2:
        return [(2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (1, 0, 1), (0, 1, 1)]
    if l == 3:
        return [(3, 0, 0), (0, 3, 0), (0, 0, 3), (1, 2, 0), (2, 1, 0),
                (2, 0, 1), (1, 0, 2), (0, 1, 2), (0, 2, 1), (1, 1, 1)]
    return [(lx, ly, l - lx - ly) for lx in range(l + 1) for ly in range(l - lx + 1)]


def _dfact(n: int) -> float:
    v = 1.0
    while n > 1:
        v *= n
        n -= 2
    return v


def primitive_norm(alpha: float, power: Tuple[int, int, int]) -> float:
    l = sum(power)
    radial = (2.0 * alpha / math.pi) ** 0.75
    ang = math.sqrt((4.0 * alpha) ** l / (_dfact(2 * power[0] - 1) * _dfact(2 * power[1] - 1)
                                         * _dfact(2 * power[2] - 1)))
    return radial * ang


def _pure_coefficient(l: int, m: int, lx: int, ly: int) -> float:
    """Schlegel-Frisch coefficient of x^lx y^ly z^lz in the real solid harmonic (l, m)."""
    f = math.factorial
    lz = l - lx - ly
    ma = abs(m)
    if ma > l or lz < 0:
        return 0.0
    j2 = l - ma - lz
    if j2 % 2:
        return 0.0
    j = j2 // 2
    a = math.sqrt(f(2 * lx) * f(2 * ly) * f(2 * lz) * f(l) / (f(2 * l) * f(lx) * f(ly) * f(lz)))
    b = math.sqrt(f(l - ma) / f(l + ma)) / (2.0 ** l * f(l))
    g = 0.0
    for i in range((l - ma) // 2 + 1):
        if j < 0 or j > i:
            continue
        c = (math.comb(l, i) * math.comb(i, j) * (-1) ** i * f(2 * l - 2 * i) / f(l - ma - 2 * i))
        for k in range(j + 1):
            if lx - 2 * k < 0 or lx - 2 * k > ma:
                continue
            d = math.comb(j, k) * math.comb(ma, lx - 2 * k)
            e = 0.0
            if m == 0 and lx % 2 == 0:
                e = (-1.0) ** (k - lx // 2)
            if m > 0 and abs(ma - lx) % 2 == 0:
                e = math.sqrt(2.0) * (-1.0) ** ((2 * k + ma - lx) // 2)
            if m < 0 and abs(ma - lx) % 2 == 1:
                e = math.sqrt(2.0) * (-1.0) ** ((2 * k + ma - lx) // 2)
            g += c * d * e
    return a * b * g


def pure_transform(l: int) -> np.ndarray:
    """(2l+1) x ncart Cartesian-to-pure matrix, rows m = 0, +1, -1, +2, -2, ..."""
    cart = cartesian_order(l)
    t = np.zeros((2 * l + 1, len(cart)))
    for g, (px, py, _) in enumerate(cart):
        t[0, g] = _pure_coefficient(l, 0, px, py)
        for m in range(1, l + 1):
            t[2 * m - 1, g] = _pure_coefficient(l, m, px, py)
            t[2 * m, g] = _pure_coefficient(l, -m, px, py)
    return t


# ---------------------------------------------------------------------------
# Molecule description
# ---------------------------------------------------------------------------


@dataclass
class ShellSpec:
    atom: int            # zero-based atom index
    l: int
    pure: bool
    exponents: np.ndarray
    coefficients: np.ndarray


@dataclass
class SyntheticMolecule:
    name: str
    atomic_numbers: np.ndarray
    coordinates: np.ndarray            # natoms x 3, bohr
    shells: List[ShellSpec]
    nalpha: int
    nbeta: int
    charge: int
    multiplicity: int
    c_alpha: np.ndarray                 # nbasis x nmo
    c_beta: Optional[np.ndarray]        # unrestricted only
    e_alpha: np.ndarray
    e_beta: Optional[np.ndarray]
    p_total: np.ndarray
    p_spin: np.ndarray
    meta: Dict[str, object] = field(default_factory=dict)

    @property
    def nbasis(self) -> int:
        return int(sum(2 * s.l + 1 if (s.pure and s.l >= 2) else (s.l + 1) * (s.l + 2) // 2
                       for s in self.shells))


def _random_shell(rng: np.random.Generator, l: int) -> Tuple[np.ndarray, np.ndarray]:
    nprim = int(rng.integers(1, 7))
    exps = np.sort(np.exp(rng.uniform(math.log(0.1), math.log(5000.0), nprim)))[::-1].copy()
    coefs = rng.uniform(0.1, 1.0, nprim)
    # Normalise the contracted x^l component: sum_pq c_p c_q S_pq = 1 with the
    # overlap of normalised primitives (2 sqrt(a b) / (a + b))^(l + 3/2).
    a = exps[:, None]
    b = exps[None, :]
    s = (2.0 * np.sqrt(a * b) / (a + b)) ** (l + 1.5)
    norm2 = float(coefs @ s @ coefs)
    return exps, coefs / math.sqrt(norm2)


def _element_basis(rng: np.random.Generator, shell_ls: Sequence[int]) -> List[Tuple[int, np.ndarray, np.ndarray]]:
    return [(l, *_random_shell(rng, l)) for l in shell_ls]


def _random_positions(rng: np.random.Generator, natoms: int, box: float, min_dist: float) -> np.ndarray:
    pos = np.zeros((natoms, 3))
    placed = 0
    attempts = 0
    while placed < natoms:
        attempts += 1
        if attempts > 2_000_000:
            raise RuntimeError("cannot place atoms with the requested spacing")
        p = rng.uniform(0.0, box, 3)
        if placed and np.min(np.linalg.norm(pos[:placed] - p, axis=1)) < min_dist:
            continue
        pos[placed] = p
        placed += 1
    return pos


# ---------------------------------------------------------------------------
# Overlap matrix (Obara-Saika, vectorised over primitive pairs)
# ---------------------------------------------------------------------------


def _blocks(shells: List[ShellSpec], coords: np.ndarray):
    """Normalised AO blocks: origin, l, exps, weights (ncart x nprim), transform, offset."""
    out = []
    off = 0
    for sh in shells:
        cart = cartesian_order(sh.l)
        w = np.array([[c * primitive_norm(a, pw) for a, c in zip(sh.exponents, sh.coefficients)]
                      for pw in cart])
        t = pure_transform(sh.l) if (sh.pure and sh.l >= 2) else np.eye(len(cart))
        out.append((coords[sh.atom], sh.l, sh.exponents, w, t, off))
        off += t.shape[0]
    return out, off


def _os_1d(la: int, lb: int, p: np.ndarray, xpa: np.ndarray, xpb: np.ndarray) -> np.ndarray:
    """1D overlap factors S_ij / S_00 for i <= la, j <= lb (last two axes)."""
    shape = p.shape
    s = np.zeros(shape + (la + 1, lb + 1))
    s[..., 0, 0] = 1.0
    h = 0.5 / p
    for i in range(la + 1):
        for j in range(lb + 1):
            if i == 0 and j == 0:
                continue
            if i > 0:
                v = xpa * s[..., i - 1, j]
                if i > 1:
                    v = v + (i - 1) * h * s[..., i - 2, j]
                if j > 0:
                    v = v + j * h * s[..., i - 1, j - 1]
            else:
                v = xpb * s[..., i, j - 1]
                if j > 1:
                    v = v + (j - 1) * h * s[..., i, j - 2]
            s[..., i, j] = v
    return s


def overlap_matrix(shells: List[ShellSpec], coords: np.ndarray, chunk: int = 4096) -> np.ndarray:
    """AO overlap matrix (Obara-Saika), vectorised over block pairs of the same
    angular momenta: exponents, weights and transforms are gathered per angular
    momentum once, and each chunk of pairs is written back with one scatter."""
    blocks, n = _blocks(shells, coords)
    S = np.zeros((n, n))
    maxp = max(len(b[2]) for b in blocks)
    by_l: Dict[int, Dict[str, np.ndarray]] = {}
    for l in sorted({b[1] for b in blocks}):
        idx = [i for i, b in enumerate(blocks) if b[1] == l]
        ncart = len(cartesian_order(l))
        exps = np.ones((len(idx), maxp))
        wts = np.zeros((len(idx), ncart, maxp))
        for r, i in enumerate(idx):
            k = len(blocks[i][2])
            exps[r, :k] = blocks[i][2]
            wts[r, :, :k] = blocks[i][3]
        t = blocks[idx[0]][4]
        if any(blocks[i][4].shape != t.shape or not np.array_equal(blocks[i][4], t) for i in idx):
            raise ValueError("blocks of one angular momentum must share their transform")
        by_l[l] = {"idx": np.array(idx), "exps": exps, "w": wts, "t": t,
                   "origin": np.array([blocks[i][0] for i in idx]),
                   "off": np.array([blocks[i][5] for i in idx])}
    ls = sorted(by_l)
    for ai, la in enumerate(ls):
        for lb in ls[ai:]:
            A_, B_ = by_l[la], by_l[lb]
            # Every unordered block pair once: all (a, b) across two angular
            # momenta, a <= b in the block order within one.
            ga, gb = np.meshgrid(np.arange(len(A_["idx"])), np.arange(len(B_["idx"])), indexing="ij")
            keep = A_["idx"][ga] <= B_["idx"][gb] if la == lb else np.ones(ga.shape, bool)
            # Pairs whose most diffuse primitives still overlap by less than
            # exp(-100) are left at zero (far below the rounding of S).
            amin = A_["exps"].min(1)[ga]
            bmin = B_["exps"].min(1)[gb]
            r2 = ((A_["origin"][ga] - B_["origin"][gb]) ** 2).sum(-1)
            keep &= amin * bmin / (amin + bmin) * r2 <= 100.0
            qa, qb = ga[keep], gb[keep]
            ca, cb = cartesian_order(la), cartesian_order(lb)
            ta, tb = A_["t"], B_["t"]
            for c0 in range(0, len(qa), chunk):
                ia, ib = qa[c0:c0 + chunk], qb[c0:c0 + chunk]
                A = A_["origin"][ia]
                B = B_["origin"][ib]
                alpha = A_["exps"][ia][:, :, None]
                beta = B_["exps"][ib][:, None, :]
                p = alpha + beta
                mu = alpha * beta / p
                s00 = np.ones_like(p) * (math.pi / p) ** 1.5
                tabs = []
                for ax in range(3):
                    ax_a = A[:, ax][:, None, None]
                    ax_b = B[:, ax][:, None, None]
                    P = (alpha * ax_a + beta * ax_b) / p
                    s00 = s00 * np.exp(-mu * (ax_a - ax_b) ** 2)
                    tabs.append(_os_1d(la, lb, p, P - ax_a, P - ax_b))
                prim = np.empty(p.shape + (len(ca), len(cb)))
                for ka, (ax, ay, az) in enumerate(ca):
                    for kb, (bx, by, bz) in enumerate(cb):
                        prim[..., ka, kb] = (s00 * tabs[0][..., ax, bx] * tabs[1][..., ay, by]
                                             * tabs[2][..., az, bz])
                cart = np.einsum("qkp,qlr,qprkl->qkl", A_["w"][ia], B_["w"][ib], prim, optimize=True)
                blk = np.einsum("ak,qkl,bl->qab", ta, cart, tb, optimize=True)
                rows = A_["off"][ia][:, None, None] + np.arange(blk.shape[1])[None, :, None]
                cols = B_["off"][ib][:, None, None] + np.arange(blk.shape[2])[None, None, :]
                S[rows, cols] = blk
                S[cols, rows] = blk
    return S


# ---------------------------------------------------------------------------
# Molecule generation
# ---------------------------------------------------------------------------

HEAVY_SHELLS = [0] * 5 + [1] * 3 + [2] * 2 + [3]      # 5s3p2d1f
HYDROGEN_SHELLS = [0] * 3 + [1]                       # 3s1p


def _orthonormal_orbitals(rng: np.random.Generator, S: np.ndarray) -> np.ndarray:
    n = S.shape[0]
    L = np.linalg.cholesky(S)
    Q, R = np.linalg.qr(rng.standard_normal((n, n)))
    Q = Q * np.sign(np.diag(R))
    # C^T S C = Q^T L^-1 L L^T L^-T Q = I.
    return np.linalg.solve(L.T, Q)


def build_molecule(name: str, elements: Sequence[str], coords: np.ndarray,
                   element_shells: Dict[str, Sequence[int]], seed: int,
                   nalpha: int, nbeta: int, charge: int = 0,
                   basis_rng: Optional[np.random.Generator] = None) -> SyntheticMolecule:
    rng = basis_rng if basis_rng is not None else np.random.default_rng(seed)
    basis_by_element = {el: _element_basis(rng, element_shells[el])
                        for el in sorted(set(elements), key=lambda e: ELEMENT_Z[e])}
    shells: List[ShellSpec] = []
    for ia, el in enumerate(elements):
        for l, e, c in basis_by_element[el]:
            shells.append(ShellSpec(ia, l, True, e.copy(), c.copy()))
    S = overlap_matrix(shells, coords)
    orb_rng = np.random.default_rng(seed + 1000)
    ca = _orthonormal_orbitals(orb_rng, S)
    unrestricted = nalpha != nbeta
    cb = _orthonormal_orbitals(orb_rng, S) if unrestricted else None
    n = S.shape[0]
    ea = np.sort(orb_rng.uniform(-20.0, 5.0, n))
    eb = np.sort(orb_rng.uniform(-20.0, 5.0, n)) if unrestricted else None
    pa = ca[:, :nalpha] @ ca[:, :nalpha].T
    pb = (cb if unrestricted else ca)[:, :nbeta] @ (cb if unrestricted else ca)[:, :nbeta].T
    z = np.array([ELEMENT_Z[e] for e in elements], dtype=np.int64)
    mult = nalpha - nbeta + 1
    return SyntheticMolecule(name, z, np.asarray(coords, dtype=float), shells, nalpha, nbeta,
                             charge, mult, ca, cb, ea, eb, pa + pb, pa - pb)


def water(seed: int = 0) -> SyntheticMolecule:
    """Closed-shell water-shaped molecule, O 4s3p1d / H 2s1p pure, 28 AOs, 5 occupied MOs."""
    coords = np.array([[0.0, 0.0, 0.2217], [0.0, 1.4309, -0.8867], [0.0, -1.4309, -0.8867]])
    shells = {"O": [0] * 4 + [1] * 3 + [2], "H": [0] * 2 + [1]}
    return build_molecule("water_28", ["O", "H", "H"], coords, shells, seed, 5, 5)


def organic(name: str, counts: Dict[str, int], seed: int, box: float, charge: int = 0,
            multiplicity: int = 1) -> SyntheticMolecule:
    rng = np.random.default_rng(seed)
    elements: List[str] = []
    for el in ("C", "N", "O", "H"):
        elements += [el] * counts.get(el, 0)
    coords = _random_positions(rng, len(elements), box, 1.8)
    nelec = sum(ELEMENT_Z[e] for e in elements) - charge
    unpaired = multiplicity - 1
    if (nelec - unpaired) % 2:
        raise ValueError("electron count and multiplicity are inconsistent")
    nbeta = (nelec - unpaired) // 2
    nalpha = nbeta + unpaired
    shells = {"C": HEAVY_SHELLS, "N": HEAVY_SHELLS, "O": HEAVY_SHELLS, "H": HYDROGEN_SHELLS}
    return build_molecule(name, elements, coords, shells, seed, nalpha, nbeta, charge, basis_rng=rng)


# The workloads.  Each entry gives the molecule and the grid (origin, spacing,
# counts along the three Cartesian axes, centred on the atoms' centroid).
WORKLOADS = {
    "water_28": dict(make=lambda: water(0), grid_n=64, spacing=0.25),
    "organic_740": dict(make=lambda: organic("organic_740", {"C": 12, "N": 4, "O": 4, "H": 20}, 1, 12.0),
                        grid_n=128, spacing=0.2),
    "triplet_3700": dict(make=lambda: organic("triplet_3700", {"C": 60, "N": 20, "O": 20, "H": 100}, 2,
                                              28.0, multiplicity=3), grid_n=192, spacing=0.17),
    # Scaled-down unrestricted triplet (same generator, seed and basis as
    # triplet_3700; 370 AOs, 39 alpha / 37 beta electrons) for parity tests
    # that the CPU oracle finishes in seconds.
    "triplet_370": dict(make=lambda: organic("triplet_370", {"C": 6, "N": 2, "O": 2, "H": 10}, 2,
                                             14.0, multiplicity=3), grid_n=96, spacing=0.17),
    # C30N3O3H24 has an odd electron count; the closed-shell molecule is its cation.
    "esp_1260": dict(make=lambda: organic("esp_1260", {"C": 30, "N": 3, "O": 3, "H": 24}, 3, 15.0,
                                          charge=1), grid_n=96, spacing=0.24),
}


def centred_grid(coords: np.ndarray, n: int, spacing: float):
    """Cube of n^3 points with the given spacing, centred on the centroid of the atoms."""
    centroid = coords.mean(axis=0)
    origin = centroid - 0.5 * spacing * (n - 1)
    return origin, np.eye(3) * spacing, (n, n, n)


# ---------------------------------------------------------------------------
# FCHK writer / reader
# ---------------------------------------------------------------------------


def _fmt_real(v: float) -> str:
    return f"{v: .16E}"


def _write_scalar(out, label: str, kind: str, value) -> None:
    if kind == "I":
        out.write(f"{label:<43}I     {int(value):12d}\n")
    else:
        out.write(f"{label:<43}R     {_fmt_real(float(value))}\n")


def _write_array(out, label: str, kind: str, values) -> None:
    values = list(values)
    out.write(f"{label:<43}{kind}   N={len(values):12d}\n")
    per = 6 if kind == "I" else 4
    for i in range(0, len(values), per):
        chunk = values[i:i + per]
        if kind == "I":
            out.write("".join(f"{int(v):12d}" for v in chunk) + "\n")
        else:
            out.write(" ".join(_fmt_real(float(v)) for v in chunk) + "\n")


def _packed_lower(m: np.ndarray) -> np.ndarray:
    n = m.shape[0]
    idx = np.tril_indices(n)
    return m[idx]


def fchk_records(mol: SyntheticMolecule) -> Dict[str, object]:
    """The FCHK records write_fchk would write, as read_fchk returns them
    (for building a molecule in memory without the file round trip)."""
    rec: Dict[str, object] = {
        "Number of atoms": len(mol.atomic_numbers),
        "Number of alpha electrons": mol.nalpha,
        "Number of beta electrons": mol.nbeta,
        "Number of basis functions": mol.nbasis,
        "Atomic numbers": np.asarray(mol.atomic_numbers, dtype=np.int64),
        "Nuclear charges": np.asarray(mol.atomic_numbers, dtype=float),
        "Current cartesian coordinates": mol.coordinates.reshape(-1),
        "Shell types": np.array([(-s.l if (s.pure and s.l >= 2) else s.l) for s in mol.shells]),
        "Number of primitives per shell": np.array([len(s.exponents) for s in mol.shells]),
        "Shell to atom map": np.array([s.atom + 1 for s in mol.shells]),
        "Primitive exponents": np.concatenate([s.exponents for s in mol.shells]),
        "Contraction coefficients": np.concatenate([s.coefficients for s in mol.shells]),
        "Coordinates of each shell": np.concatenate([mol.coordinates[s.atom] for s in mol.shells]),
        "Alpha MO coefficients": mol.c_alpha.T.reshape(-1),
        "Total SCF Density": _packed_lower(mol.p_total),
    }
    if mol.c_beta is not None:
        rec["Beta MO coefficients"] = mol.c_beta.T.reshape(-1)
    if mol.nalpha != mol.nbeta:
        rec["Spin SCF Density"] = _packed_lower(mol.p_spin)
    return rec


def serving_molecule(index: int, natoms: int, seed: int) -> SyntheticMolecule:
    """One molecule of the serving pool: natoms atoms (half heavy, C:N:O =
    3:1:1, the rest H; 3 atoms give water's composition), the same generator
    and basis as the workloads, a box at the organic workload's atom density,
    closed shell (the cation when the electron count is odd)."""
    if natoms <= 3:
        counts = {"O": 1, "H": max(0, natoms - 1)}
    else:
        heavy = max(1, natoms // 2)
        c = max(1, round(0.6 * heavy))
        nn = (heavy - c) // 2
        counts = {"C": c, "N": nn, "O": heavy - c - nn, "H": natoms - heavy}
    nelec = sum(ELEMENT_Z[e] * k for e, k in counts.items())
    box = max(6.0, 12.0 * (natoms / 40.0) ** (1.0 / 3.0))
    return organic(f"serve_{index}_{natoms}", counts, seed, box, charge=nelec % 2)


def serving_pool(count: int = 32, seed: int = 7, min_atoms: int = 3, max_atoms: int = 200) -> List[Tuple[int, int, int]]:
    """(index, atoms, seed) of the serving pool: atom counts log-uniform in
    [min_atoms, max_atoms] from a seeded generator."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(min_atoms), math.log(max_atoms + 1), count)).astype(int)
    return [(i, int(max(min_atoms, min(max_atoms, n))), seed * 1000 + i) for i, n in enumerate(sizes)]


def serving_records(spec: Tuple[int, int, int]) -> Dict[str, object]:
    """FCHK records of one serving-pool molecule (index, atoms, seed); a
    module-level function so that a process pool can build the pool."""
    index, natoms, seed = spec
    return fchk_records(serving_molecule(index, natoms, seed))


def write_fchk(mol: SyntheticMolecule, path: str) -> None:
    """Write the molecule as an FCHK file (gzip-compressed if the path ends in .gz)."""
    opener = gzip.open if path.endswith(".gz") else open
    tmp = path + ".part"
    with opener(tmp, "wt") as out:
        out.write(f"{mol.name} synthetic molecule\n")
        out.write("SP        RB3LYP                                                      Gen\n")
        _write_scalar(out, "Number of atoms", "I", len(mol.atomic_numbers))
        _write_scalar(out, "Charge", "I", mol.charge)
        _write_scalar(out, "Multiplicity", "I", mol.multiplicity)
        _write_scalar(out, "Number of electrons", "I", mol.nalpha + mol.nbeta)
        _write_scalar(out, "Number of alpha electrons", "I", mol.nalpha)
        _write_scalar(out, "Number of beta electrons", "I", mol.nbeta)
        _write_scalar(out, "Number of basis functions", "I", mol.nbasis)
        _write_scalar(out, "Number of independent functions", "I", mol.nbasis)
        _write_array(out, "Atomic numbers", "I", mol.atomic_numbers)
        _write_array(out, "Nuclear charges", "R", mol.atomic_numbers.astype(float))
        _write_array(out, "Current cartesian coordinates", "R", mol.coordinates.reshape(-1))
        types = [(-s.l if (s.pure and s.l >= 2) else s.l) for s in mol.shells]
        _write_array(out, "Shell types", "I", types)
        _write_array(out, "Number of primitives per shell", "I", [len(s.exponents) for s in mol.shells])
        _write_array(out, "Shell to atom map", "I", [s.atom + 1 for s in mol.shells])
        _write_array(out, "Primitive exponents", "R", np.concatenate([s.exponents for s in mol.shells]))
        _write_array(out, "Contraction coefficients", "R",
                     np.concatenate([s.coefficients for s in mol.shells]))
        _write_array(out, "Coordinates of each shell", "R",
                     np.concatenate([mol.coordinates[s.atom] for s in mol.shells]))
        _write_array(out, "Alpha Orbital Energies", "R", mol.e_alpha)
        if mol.e_beta is not None:
            _write_array(out, "Beta Orbital Energies", "R", mol.e_beta)
        _write_array(out, "Alpha MO coefficients", "R", mol.c_alpha.T.reshape(-1))
        if mol.c_beta is not None:
            _write_array(out, "Beta MO coefficients", "R", mol.c_beta.T.reshape(-1))
        _write_array(out, "Total SCF Density", "R", _packed_lower(mol.p_total))
        if mol.nalpha != mol.nbeta:
            _write_array(out, "Spin SCF Density", "R", _packed_lower(mol.p_spin))
    os.replace(tmp, path)


def read_fchk(path: str) -> Dict[str, object]:
    """Minimal FCHK reader: integer/real scalars and arrays, by label."""
    opener = gzip.open if open(path, "rb").read(2) == b"\x1f\x8b" else open
    with opener(path, "rt") as f:
        lines = f.read().split("\n")
    rec: Dict[str, object] = {}
    i = 2
    while i < len(lines):
        line = lines[i]
        i += 1
        if len(line) < 44:
            continue
        label = line[:43].rstrip()
        meta = line[43:].split()
        if not label or not meta or meta[0] not in ("I", "R"):
            continue
        kind = meta[0]
        conv = int if kind == "I" else (lambda t: float(t.replace("D", "E").replace("d", "E")))
        if meta[1] == "N=":
            count = int(meta[2])
            # Collect the data lines (up to the next record header, which
            # starts with a letter) and convert them in one numpy call.
            first = i
            while i < len(lines) and not lines[i][:1].isalpha():
                i += 1
            text = "\n".join(lines[first:i])
            if kind == "I":
                rec[label] = np.array(text.split(), dtype=np.int64)
            else:
                if "D" in text or "d" in text:
                    text = text.replace("D", "E").replace("d", "E")
                vals = np.fromstring(text, dtype=float, sep=" ")
                if vals.size != count:
                    raise ValueError(f"malformed real array in FCHK: {label}")
                rec[label] = vals
        else:
            rec[label] = conv(meta[1])
    return rec


def workload_fchk(name: str, cache_dir: Optional[str] = None) -> str:
    """Path of the FCHK of a workload molecule, generated on first use (cached by name)."""
    cache_dir = cache_dir or os.environ.get("KUMO_SYNTH_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "kumo_b200_synth")
    os.makedirs(cache_dir, exist_ok=True)
    path = os.path.join(cache_dir, f"{name}.fchk")
    if not os.path.exists(path):
        mol = WORKLOADS[name]["make"]()
        write_fchk(mol, path)
    return path


def workload_grid(name: str, coords: np.ndarray):
    w = WORKLOADS[name]
    return centred_grid(coords, w["grid_n"], w["spacing"])
