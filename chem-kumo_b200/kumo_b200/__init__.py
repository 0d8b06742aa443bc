"""Python binding of the B200 grid evaluator's C ABI (include/kumo_b200.h).

This module loads chem-kumo_b200/lib/libkumo_b200.so with ctypes and mirrors
chem-kumo's Evaluator API: ``Molecule.from_fchk``, ``Evaluator.evaluate`` on a
grid or at points, ``PropertyKind``/``DensityComponent`` values and the Cube
writer.  There is no CPU fallback: if the library is missing, importing the
binding raises.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "lib", "libkumo_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(os.path.dirname(HERE)), "include", "kumo_b200.h")


class PropertyKind(enum.IntEnum):
    """include/chem/kumo/evaluator.hpp:109-153 of chem-kumo."""
    Density = 0
    Gradient = 1
    Hessian = 2
    Laplacian = 3
    Tau = 4
    Orbital = 5
    Elf = 6
    ReducedGradient = 7
    SignLambda2Density = 8
    ElectrostaticPotential = 9
    Lol = 10
    InteractionRegionIndicator = 11
    DensityOverlapRegionsIndicator = 12
    HamiltonianKineticEnergy = 13
    PotentialEnergyDensity = 14
    EnergyDensity = 15
    SpinPolarization = 16
    ShannonEntropyDensity = 17
    FisherInformationDensity = 18
    AverageLocalIonizationEnergy = 19
    LocalElectronAffinity = 20
    LocalElectronAttachmentEnergy = 21
    LocalElectronegativity = 22
    LocalHardness = 23
    OrbitalGradient = 24
    OrbitalHessian = 25
    OrbitalWeightedFukuiPlus = 26
    OrbitalWeightedFukuiMinus = 27
    OrbitalWeightedFukuiZero = 28
    OrbitalWeightedDualDescriptor = 29
    TauComponents = 30
    HamiltonianKineticEnergyComponents = 31
    PotentialKineticRatio = 32
    EnergyDensityPerElectron = 33
    KineticEnergyPerElectron = 34
    ElfTsirelsonStash = 35
    LolTsirelsonStash = 36


class DensityComponent(enum.IntEnum):
    Total = 0
    Alpha = 1
    Beta = 2
    Difference = 3


class SpinChannel(enum.IntEnum):
    Alpha = 0
    Beta = 1


class Backend(enum.IntEnum):
    AUTO = 0
    AO_P = 1
    AO_MO = 2


class Precision(enum.IntEnum):
    FP64 = 0
    Mixed = 1


def channels(kind: int) -> int:
    return 3 if kind in (1, 24, 30, 31) else (6 if kind in (2, 25) else 1)


@dataclass(frozen=True)
class Property:
    kind: int
    component: int = 0
    channel: int = 0
    orbital_index: int = 0


def density(kind: PropertyKind, component: DensityComponent = DensityComponent.Total) -> Property:
    return Property(int(kind), int(component))


def orbital(index: int, channel: SpinChannel = SpinChannel.Alpha, kind: PropertyKind = PropertyKind.Orbital) -> Property:
    return Property(int(kind), 0, int(channel), index)


class KumoError(RuntimeError):
    """Error raised for a non-zero kumo_status; .status holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class InvalidArgument(KumoError, ValueError):
    pass


class OutOfRange(KumoError, IndexError):
    pass


_EXC = {1: InvalidArgument, 2: OutOfRange}


class _Property(C.Structure):
    _fields_ = [("kind", C.c_int), ("component", C.c_int), ("channel", C.c_int), ("orbital_index", C.c_longlong)]


class _Options(C.Structure):
    _fields_ = [("block_size", C.c_longlong), ("backend", C.c_int), ("screening_threshold", C.c_double),
                ("potential_tolerance", C.c_double), ("precision", C.c_int), ("fukui_delta", C.c_double)]


class _Grid(C.Structure):
    _fields_ = [("origin", C.c_double * 3), ("steps", C.c_double * 9), ("counts", C.c_int * 3)]


class _Info(C.Structure):
    _fields_ = [("natoms", C.c_int), ("nbasis", C.c_int), ("nalpha", C.c_int), ("nbeta", C.c_int),
                ("nmo_alpha", C.c_int), ("nmo_beta", C.c_int), ("unrestricted", C.c_int),
                ("ao_mo_eligible", C.c_int), ("check_errors", C.c_double * 4), ("nblocks", C.c_int),
                ("device_bytes", C.c_longlong)]


_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_lib = None

EXPORTS = [
    "kumo_default_options", "kumo_molecule_from_fchk", "kumo_molecule_from_arrays", "kumo_molecule_destroy",
    "kumo_molecule_info_get", "kumo_molecule_atoms", "kumo_molecule_block", "kumo_evaluate_grid",
    "kumo_evaluate_points", "kumo_evaluate_grid_device", "kumo_evaluate_points_device", "kumo_ao_panels",
    "kumo_screening_masks", "kumo_boys", "kumo_esp_pair_count", "kumo_esp_pairs_evaluated", "kumo_write_cube", "kumo_grid_around",
    "kumo_profile_enable", "kumo_profile_reset", "kumo_profile_read", "kumo_set_device",
    "kumo_preload_kernels", "kumo_registered_kernels",
    "kumo_evaluate_points_noalloc", "kumo_server_create", "kumo_server_destroy", "kumo_server_submit_grid",
    "kumo_server_submit_points", "kumo_server_wait", "kumo_server_drain", "kumo_server_stats_get",
    "kumo_server_reset_stats", "kumo_density_isosurface", "kumo_potential_surface", "kumo_ionization_energy_surface",
    "kumo_map_on_density_isosurface", "kumo_average_local_ionization_energy", "kumo_extract_isosurface",
    "kumo_surface_info", "kumo_surface_mesh", "kumo_surface_field", "kumo_surface_destroy",
    "kumo_surface_statistics", "kumo_write_ply", "kumo_read_cube", "kumo_cube_info", "kumo_cube_data",
    "kumo_cube_destroy", "kumo_write_cube_data", "kumo_tile_tuning_report",
]


class _SurfaceStats(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("area", "positive_area", "negative_area", "nonpolar_area", "minimum",
                                          "maximum")] + \
               [("minimum_vertex", C.c_longlong), ("maximum_vertex", C.c_longlong)] + \
               [(n, C.c_double) for n in ("average", "positive_average", "negative_average", "positive_variance",
                                          "negative_variance", "total_variance", "balance", "charge_separation",
                                          "polarity_index")] + \
               [("n_local_minima", C.c_longlong), ("n_local_maxima", C.c_longlong)]


_SCALAR_FN = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.c_longlong, C.POINTER(C.c_double), C.POINTER(C.c_double),
                         C.c_void_p)


class _ServerOptions(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_budget_bytes", C.c_double), ("max_active", C.c_int),
                ("graph_points", C.c_longlong), ("request_scratch_bytes", C.c_double), ("staging_bytes", C.c_double)]


class _ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong), ("failed", C.c_longlong),
                ("points", C.c_longlong), ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double),
                ("max_ms", C.c_double), ("busy_s", C.c_double), ("points_per_s", C.c_double),
                ("graph_captures", C.c_longlong), ("graph_replays", C.c_longlong), ("direct_runs", C.c_longlong),
                ("peak_bytes", C.c_double), ("budget_bytes", C.c_double), ("launch_s", C.c_double),
                ("copy_s", C.c_double), ("queue_ms", C.c_double)]


class _ProfileEntry(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_int), ("ms", C.c_double), ("kept_rows", C.c_double),
                ("units", C.c_double), ("flops", C.c_double), ("bytes", C.c_double)]


def lib():
    """The loaded C library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with chem-kumo_b200/build.py")
        L = C.CDLL(LIB_PATH)
        eb = [C.c_char_p, C.c_size_t]
        L.kumo_default_options.argtypes = [C.POINTER(_Options)]
        L.kumo_molecule_from_fchk.argtypes = [C.c_char_p, C.POINTER(C.c_void_p), *eb]
        L.kumo_molecule_from_arrays.argtypes = [C.c_int, _I, _D, _D, C.c_int, _I, _I, _I, _D, _D, _D, _D, C.c_int,
                                                _D, _D, C.c_int, C.c_int, _D, C.c_int, _D, C.c_int,
                                                C.POINTER(C.c_void_p), *eb]
        L.kumo_molecule_destroy.argtypes = [C.c_void_p]
        L.kumo_molecule_info_get.argtypes = [C.c_void_p, C.POINTER(_Info)]
        L.kumo_molecule_atoms.argtypes = [C.c_void_p, _I, _D, _D]
        L.kumo_molecule_block.argtypes = [C.c_void_p, C.c_int, _I, _I, _I, _I, _I, _D]
        L.kumo_evaluate_grid.argtypes = [C.c_void_p, C.POINTER(_Options), C.POINTER(_Grid), C.POINTER(_Property),
                                         C.c_int, C.POINTER(_D), _I, *eb]
        L.kumo_evaluate_points.argtypes = [C.c_void_p, C.POINTER(_Options), _D, C.c_longlong, C.POINTER(_Property),
                                           C.c_int, C.POINTER(_D), _I, *eb]
        L.kumo_evaluate_grid_device.argtypes = [C.c_void_p, C.POINTER(_Options), C.POINTER(_Grid),
                                                C.POINTER(_Property), C.c_int, C.POINTER(_D), C.c_void_p, _I, *eb]
        L.kumo_evaluate_points_device.argtypes = [C.c_void_p, C.POINTER(_Options), _D, C.c_longlong,
                                                  C.POINTER(_Property), C.c_int, C.POINTER(_D), C.c_void_p, _I, *eb]
        L.kumo_ao_panels.argtypes = [C.c_void_p, _D, C.c_int, C.c_int, C.c_int, _D, *eb]
        L.kumo_screening_masks.argtypes = [C.c_void_p, C.POINTER(_Grid), C.c_longlong, C.c_int, C.c_double,
                                           C.POINTER(C.c_ubyte), *eb]
        L.kumo_boys.argtypes = [_D, C.c_longlong, C.c_int, _D, *eb]
        L.kumo_esp_pair_count.argtypes = [C.c_void_p, C.POINTER(C.c_longlong), *eb]
        L.kumo_esp_pairs_evaluated.argtypes = [C.c_void_p, C.c_double, C.POINTER(C.c_longlong), *eb]
        L.kumo_write_cube.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(_Grid), C.c_int, _I, _D, _D, _D,
                                      C.c_longlong, *eb]
        L.kumo_grid_around.argtypes = [C.c_void_p, C.c_double, C.c_double, C.POINTER(_Grid), *eb]
        L.kumo_read_cube.argtypes = [C.c_char_p, C.POINTER(C.c_void_p), *eb]
        L.kumo_tile_tuning_report.argtypes = [C.c_char_p, C.c_size_t]
        L.kumo_tile_tuning_report.restype = C.c_longlong
        L.kumo_cube_info.argtypes = [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(_Grid), _I]
        L.kumo_cube_data.argtypes = [C.c_void_p, _I, _D, _D, _D, C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t]
        L.kumo_cube_destroy.argtypes = [C.c_void_p]
        L.kumo_cube_destroy.restype = None
        L.kumo_write_cube_data.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.POINTER(_Grid),
                                           C.c_longlong, _I, _D, _D, _D, *eb]
        L.kumo_profile_enable.argtypes = [C.c_int]
        L.kumo_set_device.argtypes = [C.c_int, *eb]
        L.kumo_preload_kernels.argtypes = [*eb]
        L.kumo_registered_kernels.argtypes = []
        L.kumo_evaluate_points_noalloc.argtypes = [C.c_void_p, C.POINTER(_Options), _D, C.c_longlong,
                                                   C.POINTER(_Property), C.c_int, C.POINTER(_D), C.c_void_p, *eb]
        L.kumo_profile_read.argtypes = [C.POINTER(_ProfileEntry), C.c_int]
        L.kumo_server_create.argtypes = [C.POINTER(_ServerOptions), C.POINTER(C.c_void_p), *eb]
        L.kumo_server_destroy.argtypes = [C.c_void_p]
        L.kumo_server_submit_grid.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(_Options), C.POINTER(_Grid),
                                              C.POINTER(_Property), C.c_int, C.POINTER(_D),
                                              C.POINTER(C.c_ulonglong), *eb]
        L.kumo_server_submit_points.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(_Options), _D, C.c_longlong,
                                                C.POINTER(_Property), C.c_int, C.POINTER(_D),
                                                C.POINTER(C.c_ulonglong), *eb]
        L.kumo_server_wait.argtypes = [C.c_void_p, C.c_ulonglong, C.c_double, _I, *eb]
        L.kumo_server_drain.argtypes = [C.c_void_p, *eb]
        L.kumo_server_stats_get.argtypes = [C.c_void_p, C.POINTER(_ServerStats), *eb]
        L.kumo_server_reset_stats.argtypes = [C.c_void_p, *eb]
        vp = C.POINTER(C.c_void_p)
        _LL = C.POINTER(C.c_longlong)
        L.kumo_density_isosurface.argtypes = [C.c_void_p, C.c_double, C.c_double, vp, *eb]
        L.kumo_potential_surface.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, vp, *eb]
        L.kumo_ionization_energy_surface.argtypes = [C.c_void_p, C.c_double, C.c_double, vp, *eb]
        L.kumo_map_on_density_isosurface.argtypes = [C.c_void_p, C.POINTER(_Options), C.POINTER(_Property), C.c_int,
                                                     C.c_double, C.c_double, vp, _I, *eb]
        L.kumo_average_local_ionization_energy.argtypes = [C.c_void_p, _D, C.c_longlong, _D, *eb]
        L.kumo_extract_isosurface.argtypes = [C.POINTER(_Grid), _D, C.c_double, _SCALAR_FN, C.c_void_p, vp, *eb]
        L.kumo_surface_info.argtypes = [C.c_void_p, _LL, _LL, _I]
        L.kumo_surface_mesh.argtypes = [C.c_void_p, _D, _LL, _I]
        L.kumo_surface_field.argtypes = [C.c_void_p, C.c_int, _D, C.POINTER(_SurfaceStats), _LL, C.c_longlong, _LL,
                                         C.c_longlong, *eb]
        L.kumo_surface_destroy.argtypes = [C.c_void_p]
        L.kumo_surface_statistics.argtypes = [_D, C.c_longlong, _LL, C.c_longlong, _D, C.c_double,
                                              C.POINTER(_SurfaceStats), _LL, C.c_longlong, _LL, C.c_longlong, *eb]
        L.kumo_write_ply.argtypes = [C.c_char_p, _D, C.c_longlong, _LL, C.c_longlong, C.POINTER(C.c_char_p),
                                     C.POINTER(_D), C.c_int, C.POINTER(C.c_char_p), C.c_int, *eb]
        _lib = L
    return _lib


def _check(status: int, err) -> None:
    if status:
        raise _EXC.get(status, KumoError)(status, err.value.decode(errors="replace"))


def _err():
    return C.create_string_buffer(512)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_D)


@dataclass
class Grid:
    """origin (3,), steps (3, 3) with steps[:, a] the step vector of axis a, counts (3,)."""
    origin: np.ndarray
    steps: np.ndarray
    counts: Tuple[int, int, int]

    @property
    def npoints(self) -> int:
        return int(np.prod(self.counts))

    def _c(self) -> _Grid:
        g = _Grid()
        for k in range(3):
            g.origin[k] = float(self.origin[k])
            g.counts[k] = int(self.counts[k])
        st = np.asarray(self.steps, dtype=float)
        for a in range(3):
            for r in range(3):
                g.steps[3 * a + r] = float(st[r, a])
        return g

    def points(self) -> np.ndarray:
        """Points in Field order (k fastest), shape (N, 3)."""
        n0, n1, n2 = self.counts
        i, j, k = np.meshgrid(np.arange(n0), np.arange(n1), np.arange(n2), indexing="ij")
        ijk = np.stack([i.ravel(), j.ravel(), k.ravel()], 1).astype(float)
        return self.origin[None, :] + ijk @ np.asarray(self.steps).T


def _options(block_size=128, backend=0, threshold=1e-12, potential_tolerance=0.0, precision=0,
             fukui_delta=0.1) -> _Options:
    return _Options(int(block_size), int(backend), float(threshold), float(potential_tolerance), int(precision),
                    float(fukui_delta))


def _props(props: Sequence[Property]):
    arr = (_Property * max(len(props), 1))()
    for i, p in enumerate(props):
        arr[i] = _Property(int(p.kind), int(p.component), int(p.channel), int(p.orbital_index))
    return arr


class Molecule:
    """Molecule::from_fchk with its device-resident copy (created on first use)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def from_fchk(cls, path: str) -> "Molecule":
        h = C.c_void_p()
        e = _err()
        _check(lib().kumo_molecule_from_fchk(path.encode(), C.byref(h), e, 512), e)
        return cls(h)

    @classmethod
    def from_records(cls, rec: Dict[str, object]) -> "Molecule":
        """From FCHK records as returned by kumo_b200.synth.read_fchk."""
        L = lib()
        z = np.ascontiguousarray(rec["Atomic numbers"], dtype=np.int32)
        charges = np.ascontiguousarray(rec.get("Nuclear charges", z.astype(float)), dtype=float)
        xyz = np.ascontiguousarray(rec["Current cartesian coordinates"], dtype=float)
        types = np.ascontiguousarray(rec["Shell types"], dtype=np.int32)
        nprim = np.ascontiguousarray(rec["Number of primitives per shell"], dtype=np.int32)
        atom = np.ascontiguousarray(rec["Shell to atom map"], dtype=np.int32)
        ex = np.ascontiguousarray(rec["Primitive exponents"], dtype=float)
        co = np.ascontiguousarray(rec["Contraction coefficients"], dtype=float)
        pc = rec.get("P(S=P) Contraction coefficients")
        pc = None if pc is None else np.ascontiguousarray(pc, dtype=float)
        sxyz = np.ascontiguousarray(rec["Coordinates of each shell"], dtype=float)
        n = int(rec["Number of basis functions"])
        pt = np.ascontiguousarray(rec["Total SCF Density"], dtype=float)
        ps = rec.get("Spin SCF Density")
        ps = None if ps is None else np.ascontiguousarray(ps, dtype=float)
        ca = np.ascontiguousarray(rec.get("Alpha MO coefficients", np.zeros(0)), dtype=float)
        cb = rec.get("Beta MO coefficients")
        cb = None if cb is None else np.ascontiguousarray(cb, dtype=float)
        h = C.c_void_p()
        e = _err()
        _check(L.kumo_molecule_from_arrays(
            len(z), z.ctypes.data_as(_I), _dp(charges), _dp(xyz), len(types), types.ctypes.data_as(_I),
            nprim.ctypes.data_as(_I), atom.ctypes.data_as(_I), _dp(ex), _dp(co), _dp(pc) if pc is not None else None,
            _dp(sxyz), n, _dp(pt), _dp(ps) if ps is not None else None, int(rec["Number of alpha electrons"]),
            int(rec["Number of beta electrons"]), _dp(ca) if ca.size else None, ca.size // n,
            _dp(cb) if cb is not None else None, 0 if cb is None else cb.size // n, C.byref(h), e, 512), e)
        return cls(h)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().kumo_molecule_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> Dict[str, object]:
        i = _Info()
        lib().kumo_molecule_info_get(self._h, C.byref(i))
        return {"natoms": i.natoms, "nbasis": i.nbasis, "nalpha": i.nalpha, "nbeta": i.nbeta,
                "nmo_alpha": i.nmo_alpha, "nmo_beta": i.nmo_beta, "unrestricted": bool(i.unrestricted),
                "ao_mo_eligible": bool(i.ao_mo_eligible), "check_errors": list(i.check_errors),
                "nblocks": i.nblocks, "device_bytes": i.device_bytes}

    def atoms(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        n = self.info()["natoms"]
        z = np.zeros(n, dtype=np.int32)
        q = np.zeros(n)
        x = np.zeros(3 * n)
        lib().kumo_molecule_atoms(self._h, z.ctypes.data_as(_I), _dp(q), _dp(x))
        return z, q, x.reshape(n, 3)

    def blocks(self) -> List[Tuple[int, int, int, int, int, float]]:
        out = []
        for i in range(self.info()["nblocks"]):
            v = [C.c_int() for _ in range(5)]
            r2 = C.c_double()
            lib().kumo_molecule_block(self._h, i, *[C.byref(x) for x in v], C.byref(r2))
            out.append(tuple(x.value for x in v) + (r2.value,))
        return out

    def grid_around(self, margin: float, spacing: float) -> Grid:
        g = _Grid()
        e = _err()
        _check(lib().kumo_grid_around(self._h, margin, spacing, C.byref(g), e, 512), e)
        st = np.zeros((3, 3))
        for a in range(3):
            for r in range(3):
                st[r, a] = g.steps[3 * a + r]
        return Grid(np.array(list(g.origin)), st, tuple(g.counts))

    # -- kernel seams --------------------------------------------------------
    def ao_panels(self, points: np.ndarray, order: int, precision: int = 0) -> np.ndarray:
        """AO panels as [panel, ao, point] (BasisEvaluator::evaluate_derivatives_batch layout transposed)."""
        pts = np.ascontiguousarray(points, dtype=float).reshape(-1, 3)
        n = self.info()["nbasis"]
        panels = 1 if order == 0 else (4 if order == 1 else 10)
        out = np.zeros((panels * len(pts), n))
        e = _err()
        _check(lib().kumo_ao_panels(self._h, _dp(pts), len(pts), order, precision, _dp(out), e, 512), e)
        return out.reshape(panels, len(pts), n).transpose(0, 2, 1).copy()

    def screening_masks(self, grid: Grid, block_size: int, ao_order: int, threshold: float) -> np.ndarray:
        n = self.info()["nbasis"]
        nb = (grid.npoints + block_size - 1) // block_size
        mask = np.zeros((nb, n), dtype=np.uint8)
        e = _err()
        g = grid._c()
        _check(lib().kumo_screening_masks(self._h, C.byref(g), block_size, ao_order, threshold,
                                          mask.ctypes.data_as(C.POINTER(C.c_ubyte)), e, 512), e)
        return mask

    def esp_pair_count(self) -> int:
        c = C.c_longlong()
        e = _err()
        _check(lib().kumo_esp_pair_count(self._h, C.byref(c), e, 512), e)
        return c.value

    def esp_pairs_evaluated(self, tolerance: float) -> int:
        """Primitive pairs evaluated for potential_tolerance `tolerance`."""
        c = C.c_longlong()
        e = _err()
        _check(lib().kumo_esp_pairs_evaluated(self._h, float(tolerance), C.byref(c), e, 512), e)
        return c.value


class Evaluator:
    """chem-kumo's Evaluator over the C ABI (host arrays in and out)."""

    def __init__(self, molecule: Molecule, block_size: int = 128, backend: int = 0, threshold: float = 1e-12,
                 potential_tolerance: float = 0.0, precision: int = 0, fukui_delta: float = 0.1):
        self.m = molecule
        self.opt = _options(block_size, backend, threshold, potential_tolerance, precision, fukui_delta)

    def _outs(self, props, n, out=None):
        if out is None:
            outs = [np.empty((channels(p.kind), n)) for p in props]
        else:
            # Caller arrays (e.g. page-locked, reused across calls): C-contiguous float64 of the right size.
            outs = list(out)
            if len(outs) != len(props):
                raise InvalidArgument(1, "one output array per property")
            for o, p in zip(outs, props):
                if (not isinstance(o, np.ndarray) or o.dtype != np.float64 or not o.flags["C_CONTIGUOUS"]
                        or o.size != channels(p.kind) * n):
                    raise InvalidArgument(1, "output arrays must be C-contiguous float64 of "
                                          "channels x points elements")
        ptrs = (_D * max(len(props), 1))(*[_dp(o) for o in outs])
        return outs, ptrs

    def evaluate_grid(self, grid: Grid, props: Sequence[Property], out=None) -> Tuple[List[np.ndarray], int]:
        outs, ptrs = self._outs(props, grid.npoints, out)
        used = C.c_int()
        e = _err()
        g = grid._c()
        _check(lib().kumo_evaluate_grid(self.m._h, C.byref(self.opt), C.byref(g), _props(props), len(props), ptrs,
                                        C.byref(used), e, 512), e)
        return outs, used.value

    def evaluate_points(self, points: np.ndarray, props: Sequence[Property], out=None) -> Tuple[List[np.ndarray], int]:
        pts = np.ascontiguousarray(points, dtype=float).reshape(-1, 3)
        outs, ptrs = self._outs(props, len(pts), out)
        used = C.c_int()
        e = _err()
        _check(lib().kumo_evaluate_points(self.m._h, C.byref(self.opt), _dp(pts), len(pts), _props(props),
                                          len(props), ptrs, C.byref(used), e, 512), e)
        return outs, used.value

    def evaluate_grid_device(self, grid: Grid, props: Sequence[Property], outputs: Sequence[int],
                             stream: int = 0) -> int:
        """outputs: device pointers (e.g. torch tensor data_ptr()), one per property."""
        ptrs = (_D * max(len(props), 1))(*[C.cast(C.c_void_p(int(o)), _D) for o in outputs])
        used = C.c_int()
        e = _err()
        g = grid._c()
        _check(lib().kumo_evaluate_grid_device(self.m._h, C.byref(self.opt), C.byref(g), _props(props), len(props),
                                               ptrs, C.c_void_p(stream), C.byref(used), e, 512), e)
        return used.value

    def evaluate_points_device(self, points_ptr: int, npoints: int, props: Sequence[Property],
                               outputs: Sequence[int], stream: int = 0) -> int:
        ptrs = (_D * max(len(props), 1))(*[C.cast(C.c_void_p(int(o)), _D) for o in outputs])
        used = C.c_int()
        e = _err()
        _check(lib().kumo_evaluate_points_device(self.m._h, C.byref(self.opt), C.cast(C.c_void_p(points_ptr), _D),
                                                 npoints, _props(props), len(props), ptrs, C.c_void_p(stream),
                                                 C.byref(used), e, 512), e)
        return used.value


def evaluate_points_noalloc(molecule: Molecule, points_ptr: int, npoints: int, props: Sequence[Property],
                            outputs: Sequence[int], stream: int = 0, block_size: int = 128,
                            threshold: float = 1e-12) -> None:
    """kumo_evaluate_points_noalloc: density properties at device points with no
    device allocation (FP64, AO-MO), for callers that cannot let the library
    call cudaMalloc.  The molecule must already have its device copy (any
    earlier evaluation of it on this device creates it); overlapping calls race
    on the library's fixed scratch array."""
    if len(outputs) != len(props):
        raise InvalidArgument(1, "one output array per property is required")
    ptrs = (_D * max(len(props), 1))(*[C.cast(C.c_void_p(int(o)), _D) for o in outputs])
    opt = _options(block_size, 0, threshold, 0.0, 0)
    e = _err()
    _check(lib().kumo_evaluate_points_noalloc(molecule._h, C.byref(opt), C.cast(C.c_void_p(points_ptr), _D),
                                              npoints, _props(props), len(props), ptrs, C.c_void_p(stream), e,
                                              512), e)


def boys(t: np.ndarray, nvalues: int) -> np.ndarray:
    t = np.ascontiguousarray(t, dtype=float).ravel()
    out = np.zeros((len(t), nvalues))
    e = _err()
    _check(lib().kumo_boys(_dp(t), len(t), nvalues, _dp(out), e, 512), e)
    return out


def write_cube(path: str, grid: Grid, z, charges, xyz, values: np.ndarray, comment: str = "Electron density",
               orbital_index: int = 0) -> None:
    z = np.ascontiguousarray(z, dtype=np.int32)
    q = np.ascontiguousarray(charges, dtype=float)
    x = np.ascontiguousarray(xyz, dtype=float).ravel()
    v = np.ascontiguousarray(values, dtype=float).ravel()
    e = _err()
    g = grid._c()
    _check(lib().kumo_write_cube(path.encode(), comment.encode(), C.byref(g), len(z), z.ctypes.data_as(_I), _dp(q),
                                 _dp(x), _dp(v), orbital_index, e, 512), e)


@dataclass
class CubeData:
    """A scalar Cube dataset (chem::kumo::CubeData): grid and atoms in bohr,
    values in Field order, the two comment lines and the header's unit."""
    grid: "Grid"
    atomic_numbers: np.ndarray
    charges: np.ndarray
    xyz: np.ndarray
    values: np.ndarray
    first_comment: str = ""
    second_comment: str = ""
    coordinates_in_angstrom: bool = False


def read_cube(path: str) -> CubeData:
    """kumo_read_cube: a scalar Cube file, plain or gzip (angstrom headers
    converted to bohr); raises KumoError with the reader's message."""
    L = lib()
    h, e = C.c_void_p(), _err()
    _check(L.kumo_read_cube(os.fsencode(path), C.byref(h), e, 512), e)
    try:
        na, g, ang = C.c_longlong(), _Grid(), C.c_int()
        L.kumo_cube_info(h, C.byref(na), C.byref(g), C.byref(ang))
        counts = tuple(int(c) for c in g.counts)
        z = np.zeros(na.value, dtype=np.int32)
        q = np.zeros(na.value)
        xyz = np.zeros((na.value, 3))
        vals = np.zeros(int(np.prod(counts)))
        c1, c2 = C.create_string_buffer(1 << 16), C.create_string_buffer(1 << 16)
        L.kumo_cube_data(h, z.ctypes.data_as(_I), _dp(q), _dp(xyz), _dp(vals), c1, len(c1), c2, len(c2))
        steps = np.array(list(g.steps)).reshape(3, 3).T  # column a = step of axis a
        grid = Grid(np.array(list(g.origin)), steps, counts)
        return CubeData(grid, z, q, xyz, vals, c1.value.decode(errors="replace"), c2.value.decode(errors="replace"),
                        bool(ang.value))
    finally:
        L.kumo_cube_destroy(h)


def write_cube_data(path: str, cube: CubeData) -> None:
    """kumo_write_cube_data: 13 significant digits, read_cube reproduces it."""
    z = np.ascontiguousarray(cube.atomic_numbers, dtype=np.int32)
    q = np.ascontiguousarray(cube.charges, dtype=float)
    x = np.ascontiguousarray(cube.xyz, dtype=float).ravel()
    v = np.ascontiguousarray(cube.values, dtype=float).ravel()
    e = _err()
    g = cube.grid._c()
    _check(lib().kumo_write_cube_data(os.fsencode(path), cube.first_comment.encode(), cube.second_comment.encode(),
                                      int(cube.coordinates_in_angstrom), C.byref(g), len(z), z.ctypes.data_as(_I),
                                      _dp(q), _dp(x), _dp(v), e, 512), e)


def tile_tuning_report() -> str:
    """The mixed form's measured tile shapes (kumo_tile_tuning_report)."""
    L = lib()
    n = L.kumo_tile_tuning_report(None, 0)
    buf = C.create_string_buffer(max(int(n), 0) + 1)
    L.kumo_tile_tuning_report(buf, len(buf))
    return buf.value.decode()


def set_device(device: int) -> None:
    e = _err()
    _check(lib().kumo_set_device(int(device), e, 512), e)


def preload_kernels() -> None:
    """Load every kernel of the library on the current device now (once per
    device); CUDA otherwise loads each kernel at its first launch."""
    e = _err()
    _check(lib().kumo_preload_kernels(e, 512), e)


def registered_kernels() -> int:
    """Kernel instantiations the library lists for preloading (no GPU needed)."""
    return int(lib().kumo_registered_kernels())


def profile_enable(on: bool = True) -> None:
    lib().kumo_profile_enable(1 if on else 0)


def profile_reset() -> None:
    lib().kumo_profile_reset()


def profile_read() -> Dict[str, Dict[str, float]]:
    arr = (_ProfileEntry * 16)()
    n = lib().kumo_profile_read(arr, 16)
    if n < 0:
        raise KumoError(3, "profile read failed")
    return {arr[i].name.decode(): {"launches": arr[i].launches, "ms": arr[i].ms, "kept_rows": arr[i].kept_rows,
                                   "units": arr[i].units, "flops": arr[i].flops, "bytes": arr[i].bytes}
            for i in range(n)}


class Server:
    """Serving loop (kumo_server_*): requests of any molecules and sizes are
    admitted in arrival order under an HBM budget and run concurrently on the
    GPU; small ones replay captured CUDA graphs.  submit_* returns a ticket and
    the output arrays the results will be written to; the molecule and the
    arrays must stay alive until wait() reports the ticket done."""

    def __init__(self, device: int = 0, hbm_budget_bytes: float = 0.0, max_active: int = 0,
                 graph_points: int = 0, request_scratch_bytes: float = 0.0, staging_bytes: float = 0.0):
        o = _ServerOptions(int(device), float(hbm_budget_bytes), int(max_active), int(graph_points),
                           float(request_scratch_bytes), float(staging_bytes))
        h = C.c_void_p()
        e = _err()
        _check(lib().kumo_server_create(C.byref(o), C.byref(h), e, 512), e)
        self._h = h
        self._keep: Dict[int, tuple] = {}

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().kumo_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        self.close()

    def _submit(self, molecule: "Molecule", props, n, evaluator_opts, grid=None, points=None, out=None):
        outs = [np.empty((channels(p.kind), n)) for p in props] if out is None else list(out)
        for o, p in zip(outs, props):
            if o.dtype != np.float64 or not o.flags["C_CONTIGUOUS"] or o.size != channels(p.kind) * n:
                raise InvalidArgument(1, "output arrays must be C-contiguous float64 of channels x points elements")
        ptrs = (_D * max(len(props), 1))(*[_dp(o) for o in outs])
        t = C.c_ulonglong()
        e = _err()
        opt = _options(**evaluator_opts)
        if grid is not None:
            g = grid._c()
            _check(lib().kumo_server_submit_grid(self._h, molecule._h, C.byref(opt), C.byref(g), _props(props),
                                                 len(props), ptrs, C.byref(t), e, 512), e)
        else:
            pts = np.ascontiguousarray(points, dtype=float).reshape(-1, 3)
            _check(lib().kumo_server_submit_points(self._h, molecule._h, C.byref(opt), _dp(pts), len(pts),
                                                   _props(props), len(props), ptrs, C.byref(t), e, 512), e)
        self._keep[t.value] = (molecule, outs)
        return t.value, outs

    def submit_grid(self, molecule: "Molecule", grid: Grid, props: Sequence[Property], out=None, **opts):
        return self._submit(molecule, props, grid.npoints, opts, grid=grid, out=out)

    def submit_points(self, molecule: "Molecule", points: np.ndarray, props: Sequence[Property], out=None, **opts):
        n = np.asarray(points).size // 3
        return self._submit(molecule, props, n, opts, points=points, out=out)

    def wait(self, ticket: int, timeout: float = 60.0) -> bool:
        done = C.c_int()
        e = _err()
        _check(lib().kumo_server_wait(self._h, ticket, float(timeout), C.byref(done), e, 512), e)
        if done.value:
            self._keep.pop(ticket, None)
        return bool(done.value)

    def drain(self) -> None:
        e = _err()
        _check(lib().kumo_server_drain(self._h, e, 512), e)
        self._keep.clear()

    def stats(self) -> Dict[str, float]:
        s = _ServerStats()
        e = _err()
        _check(lib().kumo_server_stats_get(self._h, C.byref(s), e, 512), e)
        return {name: getattr(s, name) for name, _ in _ServerStats._fields_}

    def reset_stats(self) -> None:
        e = _err()
        _check(lib().kumo_server_reset_stats(self._h, e, 512), e)


# ---------------------------------------------------------------------------
# Molecular surfaces (include/chem/kumo/surface.hpp)
# ---------------------------------------------------------------------------

HARTREE_IN_KCAL_PER_MOL = 627.5094740631
HARTREE_IN_ELECTRONVOLT = 27.211386245988


def _stats_dict(st: "_SurfaceStats", minima, maxima) -> Dict[str, object]:
    d = {name: getattr(st, name) for name, _ in _SurfaceStats._fields_}
    d["local_minima"] = [int(v) for v in minima]
    d["local_maxima"] = [int(v) for v in maxima]
    return d


@dataclass
class Surface:
    """A closed triangle mesh (bohr) with per-vertex fields and their statistics."""
    vertices: np.ndarray                 # (nv, 3)
    triangles: np.ndarray                # (nt, 3) int64, counter-clockwise seen from outside
    cells: Optional[np.ndarray] = None   # (nv, 3): grid indices of each vertex's edge's lower end
    values: List[np.ndarray] = field(default_factory=list)
    statistics: List[Dict[str, object]] = field(default_factory=list)

    def area(self) -> float:
        a, b, c = (self.vertices[self.triangles[:, i]] for i in range(3))
        return float(0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1).sum()) if len(self.triangles) else 0.0

    def volume(self) -> float:
        """Enclosed volume from the divergence theorem about the vertex centroid."""
        if not len(self.vertices):
            return 0.0
        c = self.vertices.mean(axis=0)
        a, b, d = (self.vertices[self.triangles[:, i]] - c for i in range(3))
        return float(np.einsum("ij,ij->i", a, np.cross(b, d)).sum() / 6.0)


def _take_surface(h, with_cells: bool = False) -> Surface:
    L = lib()
    try:
        nv, nt, nf = C.c_longlong(), C.c_longlong(), C.c_int()
        L.kumo_surface_info(h, C.byref(nv), C.byref(nt), C.byref(nf))
        v = np.zeros((nv.value, 3))
        t = np.zeros((nt.value, 3), dtype=np.int64)
        cells = np.zeros((nv.value, 3), dtype=np.int32) if with_cells else None
        L.kumo_surface_mesh(h, _dp(v), t.ctypes.data_as(C.POINTER(C.c_longlong)),
                            cells.ctypes.data_as(_I) if cells is not None else None)
        surf = Surface(v, t, cells)
        for i in range(nf.value):
            vals = np.zeros(nv.value)
            st = _SurfaceStats()
            e = _err()
            _check(L.kumo_surface_field(h, i, _dp(vals), C.byref(st), None, 0, None, 0, e, 512), e)
            mins = np.zeros(max(1, st.n_local_minima), dtype=np.int64)
            maxs = np.zeros(max(1, st.n_local_maxima), dtype=np.int64)
            _check(L.kumo_surface_field(h, i, None, None, mins.ctypes.data_as(C.POINTER(C.c_longlong)),
                                        st.n_local_minima, maxs.ctypes.data_as(C.POINTER(C.c_longlong)),
                                        st.n_local_maxima, e, 512), e)
            surf.values.append(vals)
            surf.statistics.append(_stats_dict(st, mins[:st.n_local_minima], maxs[:st.n_local_maxima]))
        return surf
    finally:
        L.kumo_surface_destroy(h)


def density_isosurface(m: Molecule, isovalue: float = 1e-3, spacing: float = 0.25) -> Surface:
    h, e = C.c_void_p(), _err()
    _check(lib().kumo_density_isosurface(m._h, float(isovalue), float(spacing), C.byref(h), e, 512), e)
    return _take_surface(h)


def electrostatic_potential_surface(m: Molecule, isovalue: float = 1e-3, spacing: float = 0.25,
                                    potential_tolerance: float = 1e-8) -> Surface:
    h, e = C.c_void_p(), _err()
    _check(lib().kumo_potential_surface(m._h, float(isovalue), float(spacing), float(potential_tolerance),
                                        C.byref(h), e, 512), e)
    return _take_surface(h)


def local_ionization_energy_surface(m: Molecule, isovalue: float = 1e-3, spacing: float = 0.25) -> Surface:
    h, e = C.c_void_p(), _err()
    _check(lib().kumo_ionization_energy_surface(m._h, float(isovalue), float(spacing), C.byref(h), e, 512), e)
    return _take_surface(h)


def map_on_density_isosurface(m: Molecule, props: Sequence[Property], isovalue: float = 1e-3,
                              spacing: float = 0.25, **options) -> Tuple[Surface, int]:
    h, e = C.c_void_p(), _err()
    kp = (_Property * max(1, len(props)))(*[_Property(p.kind, p.component, p.channel, p.orbital_index)
                                            for p in props])
    used = C.c_int(0)
    opt = _options(**options)
    _check(lib().kumo_map_on_density_isosurface(m._h, C.byref(opt), kp, len(props), float(isovalue), float(spacing),
                                                C.byref(h), C.byref(used), e, 512), e)
    return _take_surface(h), used.value


def average_local_ionization_energy(m: Molecule, points: np.ndarray) -> np.ndarray:
    pts = np.ascontiguousarray(points, dtype=float).reshape(-1, 3)
    out = np.zeros(len(pts))
    e = _err()
    _check(lib().kumo_average_local_ionization_energy(m._h, _dp(pts), len(pts), _dp(out), e, 512), e)
    return out


def extract_isosurface(grid: Grid, samples: np.ndarray, isovalue: float, function) -> Surface:
    """Isosurface f = isovalue of samples (Field order) on a grid; function(points (n, 3)) -> (values (n,),
    gradients (n, 3)) places the vertices."""
    samples = np.ascontiguousarray(samples, dtype=float).ravel()

    def cb(pts, n, values, grads, user):
        p = np.ctypeslib.as_array(pts, shape=(n, 3)).copy() if n else np.zeros((0, 3))
        v, g = function(p)
        if n:
            np.ctypeslib.as_array(values, shape=(n,))[:] = v
            np.ctypeslib.as_array(grads, shape=(n, 3))[:] = g

    fn = _SCALAR_FN(cb)
    h, e = C.c_void_p(), _err()
    gc = grid._c()
    _check(lib().kumo_extract_isosurface(C.byref(gc), _dp(samples), float(isovalue), fn, None, C.byref(h), e, 512), e)
    return _take_surface(h, with_cells=True)


def surface_statistics(vertices: np.ndarray, triangles: np.ndarray, values: np.ndarray,
                       polar_threshold: float = 10.0 / HARTREE_IN_KCAL_PER_MOL) -> Dict[str, object]:
    v = np.ascontiguousarray(vertices, dtype=float).reshape(-1, 3)
    t = np.ascontiguousarray(triangles, dtype=np.int64).reshape(-1, 3)
    x = np.ascontiguousarray(values, dtype=float).ravel()
    if len(x) != len(v):
        raise InvalidArgument(1, "surface values do not match the mesh vertices")
    st, e = _SurfaceStats(), _err()
    LL = C.POINTER(C.c_longlong)
    _check(lib().kumo_surface_statistics(_dp(v), len(v), t.ctypes.data_as(LL), len(t), _dp(x), float(polar_threshold),
                                         C.byref(st), None, 0, None, 0, e, 512), e)
    mins = np.zeros(max(1, st.n_local_minima), dtype=np.int64)
    maxs = np.zeros(max(1, st.n_local_maxima), dtype=np.int64)
    _check(lib().kumo_surface_statistics(_dp(v), len(v), t.ctypes.data_as(LL), len(t), _dp(x), float(polar_threshold),
                                         None, mins.ctypes.data_as(LL), st.n_local_minima, maxs.ctypes.data_as(LL),
                                         st.n_local_maxima, e, 512), e)
    return _stats_dict(st, mins[:st.n_local_minima], maxs[:st.n_local_maxima])


def write_ply(path: str, vertices: np.ndarray, triangles: np.ndarray,
              fields: Sequence[Tuple[str, np.ndarray]] = (), comments: Sequence[str] = ()) -> None:
    v = np.ascontiguousarray(vertices, dtype=float).reshape(-1, 3)
    t = np.ascontiguousarray(triangles, dtype=np.int64).reshape(-1, 3)
    arrays = [np.ascontiguousarray(a, dtype=float).ravel() for _, a in fields]
    for (name, _), a in zip(fields, arrays):
        if len(a) != len(v):
            raise InvalidArgument(1, f"PLY property '{name}' needs one value per vertex")
    names = (C.c_char_p * max(1, len(fields)))(*[n.encode() for n, _ in fields])
    vals = (_D * max(1, len(fields)))(*[_dp(a) for a in arrays])
    cs = (C.c_char_p * max(1, len(comments)))(*[c.encode() for c in comments])
    e = _err()
    _check(lib().kumo_write_ply(str(path).encode(), _dp(v), len(v), t.ctypes.data_as(C.POINTER(C.c_longlong)), len(t),
                                names, vals, len(fields), cs, len(comments), e, 512), e)
