"""ctypes loader of the CPU oracle (kumo_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker of the CUDA path and the timed CPU
baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkumo_oracle.so")

_dbl_p = C.POINTER(C.c_double)
_int_p = C.POINTER(C.c_int)


class KoProperty(C.Structure):
    _fields_ = [("kind", C.c_int), ("component", C.c_int), ("channel", C.c_int),
                ("orbital_index", C.c_long)]


class KoMolecule(C.Structure):
    _fields_ = [("basis", C.c_void_p), ("p_total", _dbl_p), ("p_spin", _dbl_p),
                ("c_alpha", _dbl_p), ("nmo_alpha", C.c_int), ("c_beta", _dbl_p),
                ("nmo_beta", C.c_int), ("nalpha", C.c_int), ("nbeta", C.c_int),
                ("ao_mo_eligible", C.c_int), ("natoms", C.c_int), ("atom_xyz", _dbl_p),
                ("atom_charge", _dbl_p)]


class KoOptions(C.Structure):
    _fields_ = [("block_size", C.c_long), ("backend", C.c_int), ("screening_threshold", C.c_double),
                ("potential_tolerance", C.c_double)]


DD_DTYPE = np.dtype([("value", "f8"), ("grad", "f8", 3), ("hess", "f8", 9), ("lap", "f8"),
                     ("tau", "f8"), ("tau_axes", "f8", 3)])

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.ko_basis_create.restype = C.c_void_p
        L.ko_basis_create.argtypes = [C.c_int, _int_p, _int_p, _dbl_p, _dbl_p, _dbl_p, _dbl_p, C.c_int,
                                      C.c_char_p, C.c_int]
        L.ko_basis_destroy.argtypes = [C.c_void_p]
        L.ko_basis_nao.argtypes = [C.c_void_p]
        L.ko_basis_nblocks.argtypes = [C.c_void_p]
        L.ko_basis_block.argtypes = [C.c_void_p, C.c_int, _int_p, _int_p, _int_p, _int_p, _int_p, _dbl_p]
        L.ko_pure_transform.argtypes = [C.c_int, _dbl_p]
        L.ko_primitive_norm.restype = C.c_double
        L.ko_primitive_norm.argtypes = [C.c_double, C.c_int, C.c_int, C.c_int]
        L.ko_ao_values_batch.argtypes = [C.c_void_p, _dbl_p, C.c_int, _dbl_p]
        L.ko_ao_derivatives_batch.argtypes = [C.c_void_p, _dbl_p, C.c_int, C.c_int, _dbl_p]
        L.ko_significant_aos.argtypes = [_dbl_p, C.c_int, C.c_long, C.c_double, C.POINTER(C.c_ubyte)]
        L.ko_evaluate.argtypes = [C.POINTER(KoMolecule), C.POINTER(KoOptions), _dbl_p, _dbl_p, _int_p,
                                  _dbl_p, C.c_long, C.POINTER(KoProperty), C.c_int,
                                  C.POINTER(_dbl_p), _int_p, C.c_char_p, C.c_int]
        L.ko_density_derivatives_mo.argtypes = [C.POINTER(KoMolecule), _dbl_p, C.c_long, C.c_long,
                                                C.c_int, C.c_double, C.c_void_p * 4]
        L.ko_density_derivatives_shared.argtypes = [C.POINTER(KoMolecule), _dbl_p, C.c_long, C.c_long,
                                                    C.c_int, C.c_double, C.c_void_p * 4]
        L.ko_validate_orbital_backend.argtypes = [C.c_int, _dbl_p, _dbl_p, _dbl_p, C.c_int, _dbl_p,
                                                  C.c_int, C.c_int, C.c_int, C.c_int, _dbl_p]
        L.ko_grid_points.argtypes = [_dbl_p, _dbl_p, _int_p, C.c_long, C.c_long, _dbl_p]
        L.ko_boys.argtypes = [C.c_double, C.c_int, _dbl_p]
        L.ko_esp_create.restype = C.c_void_p
        L.ko_esp_create.argtypes = [C.c_void_p, _dbl_p, C.c_int, _dbl_p, _dbl_p]
        L.ko_esp_destroy.argtypes = [C.c_void_p]
        L.ko_esp_pair_count.restype = C.c_long
        L.ko_esp_pair_count.argtypes = [C.c_void_p]
        L.ko_esp_evaluate.argtypes = [C.c_void_p, _dbl_p, C.c_long, _dbl_p]
        L.ko_esp_nuclear.argtypes = [C.c_void_p, _dbl_p, C.c_long, _dbl_p]
        L.ko_set_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dbl_p)


def _ip(a: np.ndarray):
    return a.ctypes.data_as(_int_p)


def unpack_lower(packed: np.ndarray, n: int) -> np.ndarray:
    """Packed lower triangle (row-major, i >= j), src/molecule.cpp:20-33."""
    m = np.zeros((n, n))
    idx = np.tril_indices(n)
    m[idx] = packed
    m.T[idx] = packed
    return m


class OracleMolecule:
    """Molecule loaded from FCHK records for the CPU oracle."""

    def __init__(self, rec: Dict[str, object]):
        L = lib()
        self.rec = rec
        n = int(rec["Number of basis functions"])
        self.n = n
        types = np.ascontiguousarray(rec["Shell types"], dtype=np.int32)
        nprim = np.ascontiguousarray(rec["Number of primitives per shell"], dtype=np.int32)
        self.exps = np.ascontiguousarray(rec["Primitive exponents"], dtype=float)
        self.coefs = np.ascontiguousarray(rec["Contraction coefficients"], dtype=float)
        pc = rec.get("P(S=P) Contraction coefficients")
        self.pcoefs = None if pc is None else np.ascontiguousarray(pc, dtype=float)
        self.shell_xyz = np.ascontiguousarray(rec["Coordinates of each shell"], dtype=float)
        err = C.create_string_buffer(256)
        self.basis = L.ko_basis_create(len(types), _ip(types), _ip(nprim), _p(self.exps), _p(self.coefs),
                                       _p(self.pcoefs) if self.pcoefs is not None else None,
                                       _p(self.shell_xyz), n, err, 256)
        if not self.basis:
            raise RuntimeError(err.value.decode())
        self.p_total = np.ascontiguousarray(unpack_lower(np.asarray(rec["Total SCF Density"]), n))
        if "Spin SCF Density" in rec:
            self.p_spin = np.ascontiguousarray(unpack_lower(np.asarray(rec["Spin SCF Density"]), n))
        else:
            self.p_spin = np.zeros((n, n))
        self.nalpha = int(rec["Number of alpha electrons"])
        self.nbeta = int(rec["Number of beta electrons"])
        ca = np.asarray(rec.get("Alpha MO coefficients", np.zeros(0)), dtype=float)
        cb = rec.get("Beta MO coefficients")
        self.c_alpha = np.ascontiguousarray(ca)
        self.nmo_alpha = ca.size // n
        self.c_beta = None if cb is None else np.ascontiguousarray(np.asarray(cb, dtype=float))
        self.nmo_beta = 0 if cb is None else self.c_beta.size // n
        self.unrestricted = self.c_beta is not None
        z = np.asarray(rec["Atomic numbers"])
        self.atom_xyz = np.ascontiguousarray(rec["Current cartesian coordinates"], dtype=float)
        self.atom_charge = np.ascontiguousarray(rec.get("Nuclear charges", z.astype(float)), dtype=float)
        self.natoms = len(z)
        errs = np.zeros(4)
        self.eligible = bool(self.nmo_alpha >= self.nalpha and (not self.unrestricted or self.nmo_beta >= self.nbeta)
                             and L.ko_validate_orbital_backend(
                                 n, _p(self.p_total), _p(self.p_spin), _p(self.c_alpha), self.nmo_alpha,
                                 _p(self.c_beta) if self.c_beta is not None else None, self.nmo_beta,
                                 self.nalpha, self.nbeta, int(self.unrestricted), _p(errs)))
        self.check_errors = errs
        self._km = KoMolecule(self.basis, _p(self.p_total), _p(self.p_spin), _p(self.c_alpha), self.nmo_alpha,
                              _p(self.c_beta) if self.c_beta is not None else None, self.nmo_beta,
                              self.nalpha, self.nbeta, int(self.eligible), self.natoms, _p(self.atom_xyz),
                              _p(self.atom_charge))

    @classmethod
    def from_fchk(cls, path: str) -> "OracleMolecule":
        import sys
        sys.path.insert(0, os.path.join(os.path.dirname(HERE), "chem-kumo_b200"))
        from kumo_b200.synth import read_fchk
        return cls(read_fchk(path))

    def __del__(self):
        if getattr(self, "basis", None):
            lib().ko_basis_destroy(self.basis)
            self.basis = None

    # -- AO kernels ----------------------------------------------------------
    def blocks(self) -> List[Tuple[int, int, int, int, int, float]]:
        L = lib()
        out = []
        for i in range(L.ko_basis_nblocks(self.basis)):
            v = [C.c_int() for _ in range(5)]
            r2 = C.c_double()
            L.ko_basis_block(self.basis, i, *[C.byref(x) for x in v], C.byref(r2))
            out.append(tuple(x.value for x in v) + (r2.value,))
        return out

    def ao_values(self, pts: np.ndarray) -> np.ndarray:
        pts = np.ascontiguousarray(pts, dtype=float).reshape(-1, 3)
        out = np.zeros((len(pts), self.n))  # column-major nao x b == row-major b x nao
        lib().ko_ao_values_batch(self.basis, _p(pts), len(pts), _p(out))
        return out.T.copy()

    def ao_derivatives(self, pts: np.ndarray, order: int) -> np.ndarray:
        """Panels as an array [panel, ao, point]."""
        pts = np.ascontiguousarray(pts, dtype=float).reshape(-1, 3)
        panels = 10 if order == 2 else 4
        out = np.zeros((panels * len(pts), self.n))
        lib().ko_ao_derivatives_batch(self.basis, _p(pts), len(pts), order, _p(out))
        return out.reshape(panels, len(pts), self.n).transpose(0, 2, 1).copy()

    # -- evaluator -----------------------------------------------------------
    def evaluate(self, props: Sequence[Tuple[int, int, int, int]], *, grid=None, points=None,
                 block_size: int = 128, backend: int = 0, threshold: float = 1e-12,
                 threads: int = 0) -> Tuple[List[np.ndarray], int]:
        """props: (kind, component, channel, orbital_index). Returns per-property
        arrays [channels, npts] and the backend used (1 AO_P, 2 AO_MO)."""
        L = lib()
        if threads:
            L.ko_set_threads(threads)
        if grid is not None:
            origin, steps, counts = grid
            origin = np.ascontiguousarray(origin, dtype=float)
            steps_cm = np.ascontiguousarray(np.asarray(steps, dtype=float).T)  # column a contiguous
            counts = np.ascontiguousarray(counts, dtype=np.int32)
            npts = int(np.prod(counts))
            pts_p = None
        else:
            pts = np.ascontiguousarray(points, dtype=float).reshape(-1, 3)
            npts = len(pts)
        kp = (KoProperty * len(props))(*[KoProperty(*p) for p in props])
        outs = [np.zeros((_channels(p[0]), npts)) for p in props]
        optr = (_dbl_p * len(props))(*[_p(o) for o in outs])
        opt = KoOptions(block_size, backend, threshold, 0.0)
        used = C.c_int(0)
        err = C.create_string_buffer(256)
        if grid is not None:
            st = L.ko_evaluate(C.byref(self._km), C.byref(opt), _p(origin), _p(steps_cm), _ip(counts), None,
                               0, kp, len(props), optr, C.byref(used), err, 256)
        else:
            st = L.ko_evaluate(C.byref(self._km), C.byref(opt), None, None, None, _p(pts), npts, kp,
                               len(props), optr, C.byref(used), err, 256)
        if st:
            raise ValueError(err.value.decode())
        return outs, used.value

    def density_derivatives(self, pts: np.ndarray, components: Sequence[int], ao_order: int = 2,
                            backend: str = "mo", block: int = 128, threshold: float = 1e-12) -> Dict[int, np.ndarray]:
        pts = np.ascontiguousarray(pts, dtype=float).reshape(-1, 3)
        res = {c: np.zeros(len(pts), dtype=DD_DTYPE) for c in components}
        arr = (C.c_void_p * 4)(*[res[c].ctypes.data if c in res else None for c in range(4)])
        fn = lib().ko_density_derivatives_mo if backend == "mo" else lib().ko_density_derivatives_shared
        st = fn(C.byref(self._km), _p(pts), len(pts), block, ao_order, threshold, arr)
        if st:
            raise ValueError(f"oracle density derivatives failed ({st})")
        return res


# -- orbital-energy fields ------------------------------------------------------
ORBITAL_ENERGY_KINDS = (19, 20, 21, 22, 23, 26, 27, 28, 29)


def _fukui_weights(e: np.ndarray, mu: float, delta: float) -> np.ndarray:
    """Normalized Gaussian weights (src/orbital_energy_fields.hpp:77-97)."""
    x = -((mu - e) / delta) ** 2
    g = np.exp(x - x.max())
    return g / g.sum()


def orbital_energy_fields(mol: OracleMolecule, pts: np.ndarray, kinds: Sequence[int],
                          fukui_delta: float = 0.1) -> List[np.ndarray]:
    """ALIE, LEA, LEAE, local electronegativity and hardness, and the
    orbital-weighted Fukui functions at `pts` [N, 3]: the orbital sums of
    src/orbital_energy_fields.hpp:145-264 over the AO values of every shell
    (evaluate_batch), then the fields of src/evaluator.cpp:480-516."""
    n = mol.n
    rec = mol.rec
    phi = mol.ao_values(pts)  # [nao, N]
    ca = mol.c_alpha.reshape(mol.nmo_alpha, n).T
    ea = np.asarray(rec["Alpha Orbital Energies"], dtype=float)
    na, nb = mol.nalpha, mol.nbeta
    occ, occ_e, vir, vir_e, att, att_e = [], [], [], [], [], []

    def channel(c, e, occupied, doubly, weight):
        for i in range(c.shape[1]):
            if i < occupied:
                occ.append(np.sqrt(2.0 if i < doubly else 1.0) * c[:, i])
                occ_e.append(abs(e[i]))
            else:
                vir.append(c[:, i])
                vir_e.append(e[i])
                if e[i] < 0.0:
                    att.append(np.sqrt(weight) * c[:, i])
                    att_e.append(e[i])

    if mol.unrestricted:
        cb = mol.c_beta.reshape(mol.nmo_beta, n).T
        eb = np.asarray(rec["Beta Orbital Energies"], dtype=float)
        channel(ca, ea, na, 0, 1.0)
        channel(cb, eb, nb, 0, 1.0)
    else:
        channel(ca, ea, max(na, nb), min(na, nb), 2.0)

    def sums(cols, energies):
        if not cols:
            return np.zeros(phi.shape[1]), np.zeros(phi.shape[1])
        x2 = (np.array(cols) @ phi) ** 2
        return x2.sum(0), np.asarray(energies) @ x2

    rho, e_occ = sums(occ, occ_e)
    d_vir, e_vir = sums(vir, vir_e)
    _, e_att = sums(att, att_e)
    with np.errstate(divide="ignore", invalid="ignore"):
        alie = np.where(rho > 0, e_occ / rho, 0.0)
        lea = np.where(d_vir > 0, -e_vir / d_vir, 0.0)
        attach = np.where(rho > 0, e_att / rho, 0.0)
    plus = minus = np.zeros(phi.shape[1])
    if any(k >= 26 for k in kinds):
        mu = 0.5 * (ea[na - 1] + ea[na])
        gp = _fukui_weights(ea[na:], mu, fukui_delta)
        gm = _fukui_weights(ea[:na], mu, fukui_delta)
        plus = gp @ ((ca[:, na:].T @ phi) ** 2)
        minus = gm @ ((ca[:, :na].T @ phi) ** 2)
    table = {19: alie, 20: lea, 21: attach, 22: 0.5 * (alie + lea), 23: 0.5 * (alie - lea),
             26: plus, 27: minus, 28: 0.5 * (plus + minus), 29: plus - minus}
    return [table[k].copy() for k in kinds]


def _channels(kind: int) -> int:
    return 3 if kind in (1, 24, 30, 31) else (6 if kind in (2, 25) else 1)


def grid_points(origin, steps, counts) -> np.ndarray:
    """Points of a grid in Field order (k fastest), src/grid_geometry.hpp:59-86."""
    origin = np.ascontiguousarray(origin, dtype=float)
    steps_cm = np.ascontiguousarray(np.asarray(steps, dtype=float).T)
    counts = np.ascontiguousarray(counts, dtype=np.int32)
    n = int(np.prod(counts))
    out = np.zeros((n, 3))
    lib().ko_grid_points(_p(origin), _p(steps_cm), _ip(counts), 0, n, _p(out))
    return out


def boys(t: float, nvalues: int) -> np.ndarray:
    out = np.zeros(nvalues)
    if lib().ko_boys(float(t), nvalues, _p(out)):
        raise ValueError("invalid Boys function argument")
    return out


class OracleESP:
    def __init__(self, mol: OracleMolecule):
        self.mol = mol
        self.h = lib().ko_esp_create(mol.basis, _p(mol.p_total), mol.natoms, _p(mol.atom_xyz), _p(mol.atom_charge))

    def __del__(self):
        if getattr(self, "h", None):
            lib().ko_esp_destroy(self.h)
            self.h = None

    @property
    def pair_count(self) -> int:
        return lib().ko_esp_pair_count(self.h)

    def evaluate(self, pts: np.ndarray) -> np.ndarray:
        pts = np.ascontiguousarray(pts, dtype=float).reshape(-1, 3)
        out = np.zeros(len(pts))
        lib().ko_esp_evaluate(self.h, _p(pts), len(pts), _p(out))
        return out
