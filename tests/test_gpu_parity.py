"""Parity of the CUDA path (through the C ABI) with the CPU oracle and with
chem-kumo's golden data.  Tolerances: FP64 fields within 1e-12 of the oracle
in the scaled metric max|gpu - ref| / max(1, max|ref|)
(tests/density_screening_test.cpp:137-150 of chem-kumo); screening masks and
point order bit-exact; mixed precision within 1e-7 of FP64 in the same
metric."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_points, scaled_error

import kumo_b200 as K
from kumo_b200 import synth
import oracle as O

pytestmark = pytest.mark.gpu

P = K.PropertyKind
D = K.DensityComponent


@pytest.fixture(scope="module")
def water28(tmp_path_factory):
    path = str(tmp_path_factory.mktemp("w") / "water_28.fchk")
    synth.write_fchk(synth.water(0), path)
    return path


def _pair(path):
    return K.Molecule.from_fchk(path), O.OracleMolecule.from_fchk(path)


def _box_points(xyz, n, seed, margin=2.5):
    rng = np.random.default_rng(seed)
    lo, hi = xyz.min(0) - margin, xyz.max(0) + margin
    pts = rng.uniform(lo, hi, (n, 3))
    pts[: len(xyz)] = xyz  # include the nuclei themselves
    return pts


@pytest.mark.parametrize("name", ["o2.fchk.gz", "h2o_b3lyp_def2tzvp.fchk.gz", "acrolein.fchk.gz"])
def test_ao_panels_fp64(name):
    m, o = _pair(os.path.join(GOLDEN, name))
    pts = _box_points(o.atom_xyz.reshape(-1, 3), 128, 1)
    for order in (0, 1, 2):
        g = m.ao_panels(pts, order)
        r = o.ao_values(pts)[None] if order == 0 else o.ao_derivatives(pts, order)
        scale = np.maximum(np.abs(r), 1e-300)
        rel = np.abs(g - r) / scale
        # Same operation order as the oracle: differences only where CUDA's
        # exp and the host libm differ in the last bit.
        assert np.mean(g == r) > 0.8
        assert np.max(rel[np.abs(r) > 1e-280]) < 1e-13
        assert np.array_equal(g == 0.0, r == 0.0)  # cutoff zeros identical


@pytest.mark.parametrize("name", ["o2.fchk.gz", "h2o_b3lyp_def2tzvp.fchk.gz", "acrolein.fchk.gz"])
def test_ao_panels_mixed_fp32(name):
    # FP32 AO build of the mixed form (factorised radial sums): each panel row
    # within FP32 accuracy of the oracle's FP64 values, relative to the row's
    # largest magnitude; cutoff zeros identical.
    m, o = _pair(os.path.join(GOLDEN, name))
    pts = _box_points(o.atom_xyz.reshape(-1, 3), 128, 3)
    for order in (0, 1, 2):
        g = m.ao_panels(pts, order, precision=1)
        r = o.ao_values(pts)[None] if order == 0 else o.ao_derivatives(pts, order)
        scale = np.maximum(np.abs(r).max(axis=2, keepdims=True), 1e-300)
        assert np.max(np.abs(g - r) / scale) < 2e-6, (order, np.max(np.abs(g - r) / scale))
        assert np.all(g[r == 0.0] == 0.0)  # cutoff zeros stay exact zeros
        assert np.all(np.abs(r[(g == 0.0) & (r != 0.0)]) < 1e-30)  # FP32 underflow only


@pytest.mark.parametrize("order,thr", [(0, 1e-12), (1, 1e-12), (2, 1e-12), (2, 1e-3), (2, 0.0)])
def test_screening_masks_bit_exact(order, thr):
    path = os.path.join(GOLDEN, "acrolein.fchk.gz")
    m, o = _pair(path)
    grid = m.grid_around(2.0, 0.45)
    gm = m.screening_masks(grid, 128, order, thr)
    pts = grid.points()
    for b in range(gm.shape[0]):
        blk = pts[b * 128:(b + 1) * 128]
        if order == 0:
            panels = o.ao_values(blk)[None]
        else:
            panels = o.ao_derivatives(blk, order)
        mx = np.abs(panels).max(axis=(0, 2))
        ref = np.ones(o.n, bool) if thr == 0.0 else mx > thr
        assert np.array_equal(gm[b].astype(bool), ref), f"block {b}"


FIELDS = [(P.Density, D.Total), (P.Gradient, D.Total), (P.Laplacian, D.Total), (P.Tau, D.Total), (P.Elf, D.Total)]


def _compare(outs, refs, tol, props):
    for p, a, r in zip(props, outs, refs):
        err = scaled_error(a, r)
        assert err <= tol, f"{p}: {err}"


def test_water28_fields_full_grid(water28):
    """Config 0 workload: rho, grad rho, lap rho (and tau, ELF) on the 64^3 grid."""
    m, o = _pair(water28)
    origin, steps, counts = synth.workload_grid("water_28", o.atom_xyz.reshape(-1, 3))
    grid = K.Grid(origin, steps, counts)
    props = [K.density(k, c) for k, c in FIELDS]
    outs, used = K.Evaluator(m).evaluate_grid(grid, props)
    refs, rused = o.evaluate([(int(p.kind), int(p.component), 0, 0) for p in props], grid=(origin, steps, counts))
    assert used == rused == 2
    _compare(outs[:4], refs[:4], 1e-12, props[:4])
    # ELF is a ratio of small quantities in the low-density tails, where the
    # 1e-16 rounding of the contraction order is amplified.
    dense = refs[0][0] > 1e-6
    assert scaled_error(outs[4][:, dense], refs[4][:, dense]) <= 1e-10
    assert scaled_error(outs[4], refs[4]) <= 1e-10


ALL_DENSITY = [(P.Density, D.Total), (P.Density, D.Alpha), (P.Density, D.Beta), (P.Density, D.Difference),
               (P.Gradient, D.Total), (P.Gradient, D.Alpha), (P.Hessian, D.Total), (P.Hessian, D.Beta),
               (P.Laplacian, D.Total), (P.Laplacian, D.Difference), (P.Tau, D.Total), (P.Tau, D.Beta),
               (P.Elf, D.Total), (P.Elf, D.Alpha), (P.ReducedGradient, D.Total), (P.SignLambda2Density, D.Total),
               (P.Lol, D.Total), (P.Lol, D.Beta), (P.InteractionRegionIndicator, D.Total),
               (P.DensityOverlapRegionsIndicator, D.Total), (P.HamiltonianKineticEnergy, D.Total),
               (P.PotentialEnergyDensity, D.Total), (P.EnergyDensity, D.Total), (P.SpinPolarization, D.Difference),
               (P.ShannonEntropyDensity, D.Total), (P.FisherInformationDensity, D.Total), (P.TauComponents, D.Alpha),
               (P.HamiltonianKineticEnergyComponents, D.Total), (P.PotentialKineticRatio, D.Total),
               (P.EnergyDensityPerElectron, D.Total), (P.KineticEnergyPerElectron, D.Total),
               (P.ElfTsirelsonStash, D.Total), (P.LolTsirelsonStash, D.Beta)]


@pytest.mark.parametrize("backend", [K.Backend.AO_MO, K.Backend.AO_P])
@pytest.mark.parametrize("name", ["o2.fchk.gz", "h2o_b3lyp_def2tzvp.fchk.gz"])
def test_all_density_properties(name, backend):
    m, o = _pair(os.path.join(GOLDEN, name))
    grid = m.grid_around(2.0, 0.5)
    props = [K.density(k, c) for k, c in ALL_DENSITY]
    tuples = [(int(p.kind), int(p.component), 0, 0) for p in props]
    outs, used = K.Evaluator(m, backend=backend).evaluate_grid(grid, props)
    refs, rused = o.evaluate(tuples, grid=(grid.origin, grid.steps, grid.counts), backend=int(backend))
    assert used == rused == int(backend)
    for p, a, r in zip(props, outs, refs):
        if p.kind == P.SignLambda2Density:
            # The sign of lambda2 is rounding-dependent only where lambda2 ~ 0.
            close = np.isclose(a, r, rtol=1e-10, atol=1e-12)
            assert np.mean(close) > 0.999 and np.array_equal(np.abs(a) > 0, np.abs(r) > 0)
            assert scaled_error(np.abs(a), np.abs(r)) <= 1e-12
            continue
        tol = 1e-12
        if p.kind in (P.Elf, P.Lol, P.ElfTsirelsonStash, P.LolTsirelsonStash, P.ReducedGradient,
                      P.InteractionRegionIndicator, P.DensityOverlapRegionsIndicator, P.SpinPolarization,
                      P.PotentialKineticRatio, P.EnergyDensityPerElectron, P.KineticEnergyPerElectron):
            # Ratios of small densities amplify the 1e-16 rounding of the
            # contraction order in the low-density tails; compare where the
            # density is not negligible.
            rho = refs[0][0]
            mask = rho > 1e-6
            a, r = a[:, mask], r[:, mask]
            tol = 1e-9
        assert scaled_error(a, r) <= tol, f"{p}: {scaled_error(a, r)}"


TRIPLET_FIELDS = [(P.Density, D.Alpha), (P.Density, D.Beta), (P.Density, D.Difference), (P.Density, D.Total),
                  (P.ReducedGradient, D.Total), (P.SignLambda2Density, D.Total), (P.Hessian, D.Total)]


def _grid_blocks(grid, nblocks):
    """Points of nblocks evenly spaced 128-point blocks of a grid (block structure kept)."""
    pts = grid.points()
    nb = (len(pts) + 127) // 128
    pick = np.unique(np.linspace(0, nb - 1, nblocks).astype(int))
    return np.concatenate([pts[b * 128:(b + 1) * 128] for b in pick])


@pytest.mark.parametrize("backend", [K.Backend.AO_MO, K.Backend.AO_P])
def test_unrestricted_triplet_rdg_sign_lambda2(synth_cache, backend):
    # The unrestricted-triplet workload's path (alpha, beta and spin densities,
    # RDG and sign(lambda2) rho from the full AO Hessian, screening threshold
    # 1e-10) on the scaled-down molecule of the same generator: FP64 against
    # the oracle on blocks spread over its 96^3 grid.
    path = synth.workload_fchk("triplet_370", synth_cache)
    m, o = _pair(path)
    origin, steps, counts = synth.workload_grid("triplet_370", m.atoms()[2])
    pts = _grid_blocks(K.Grid(origin, steps, counts), 48)
    props = [K.density(k, c) for k, c in TRIPLET_FIELDS]
    tuples = [(int(p.kind), int(p.component), 0, 0) for p in props]
    outs, used = K.Evaluator(m, backend=backend, threshold=1e-10).evaluate_points(pts, props)
    refs, rused = o.evaluate(tuples, points=pts, backend=int(backend), threshold=1e-10)
    assert used == rused == int(backend)
    rho = refs[3][0]
    for p, a, r in zip(props, outs, refs):
        if p.kind == P.SignLambda2Density:
            assert np.mean(np.isclose(a, r, rtol=1e-10, atol=1e-12)) > 0.999
            assert scaled_error(np.abs(a), np.abs(r)) <= 1e-12
        elif p.kind == P.ReducedGradient:
            mask = rho > 1e-6
            assert scaled_error(a[:, mask], r[:, mask]) <= 1e-9, p
        else:
            assert scaled_error(a, r) <= 1e-12, (p, scaled_error(a, r))


def test_unrestricted_triplet_mixed(synth_cache):
    # Mixed form on the same blocks: alpha and beta channels with 39 and 37
    # occupied MOs, full Hessian (10 panels, two MO passes of the tensor-core
    # contraction per channel).
    path = synth.workload_fchk("triplet_370", synth_cache)
    m = K.Molecule.from_fchk(path)
    origin, steps, counts = synth.workload_grid("triplet_370", m.atoms()[2])
    pts = _grid_blocks(K.Grid(origin, steps, counts), 48)
    props = [K.density(k, c) for k, c in TRIPLET_FIELDS if k != P.SignLambda2Density]
    f64, _ = K.Evaluator(m, threshold=1e-10).evaluate_points(pts, props)
    mix, _ = K.Evaluator(m, threshold=1e-10, precision=K.Precision.Mixed).evaluate_points(pts, props)
    total = f64[3]
    for p, a, r in zip(props, mix, f64):
        if p.kind == P.ReducedGradient:
            mask = total[0] > 1e-3
            err = np.abs(a[:, mask] - r[:, mask]).max() / max(1.0, np.abs(r[:, mask]).max())
            assert err <= 1e-5, (p, err)
            continue
        scale = max(1.0, np.abs(total).max()) if p.component == D.Difference else max(1.0, np.abs(r).max())
        assert np.abs(a - r).max() / scale <= 1e-6, p


@pytest.mark.parametrize("block", [1, 7, 32, 37, 128, 129, 200, 256, 1000, 65536])
@pytest.mark.parametrize("backend", [K.Backend.AO_MO, K.Backend.AO_P])
def test_block_sizes(block, backend):
    # Screening blocks of any size of chem-kumo's EvaluationOptions::block_size
    # (1..65536, include/chem/kumo/evaluator.hpp:411): above 128 points the
    # device screens each block over all of its 128-point chunks.  The grid
    # request takes the point path (rho, gradient, Laplacian) and, for AO-P,
    # the grid path of the alpha density (src/density.cpp:366-444).
    m, o = _pair(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    grid = m.grid_around(1.5, 0.6)
    props = [K.density(P.Density), K.density(P.Gradient), K.density(P.Laplacian), K.density(P.Density, D.Alpha)]
    tuples = [(int(p.kind), int(p.component), 0, 0) for p in props]
    outs, used = K.Evaluator(m, block_size=block, backend=backend).evaluate_grid(grid, props)
    refs, rused = o.evaluate(tuples, grid=(grid.origin, grid.steps, grid.counts), block_size=block,
                             backend=int(backend))
    assert used == rused == int(backend)
    _compare(outs, refs, 1e-12, props)
    pts = grid.points()[::5]
    outs, _ = K.Evaluator(m, block_size=block, backend=backend, threshold=1e-6).evaluate_points(pts, props)
    refs, _ = o.evaluate(tuples, points=pts, block_size=block, backend=int(backend), threshold=1e-6)
    _compare(outs, refs, 1e-12, props)


@pytest.mark.parametrize("block,thr", [(200, 1e-12), (384, 1e-6), (1000, 1e-3), (300, 0.0)])
def test_screening_masks_large_blocks(block, thr):
    m, o = _pair(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    grid = m.grid_around(2.0, 0.45)
    gm = m.screening_masks(grid, block, 2, thr)
    pts = grid.points()
    assert gm.shape[0] == (len(pts) + block - 1) // block
    for b in range(gm.shape[0]):
        blk = pts[b * block:(b + 1) * block]
        mx = np.abs(o.ao_derivatives(blk, 2)).max(axis=(0, 2))
        ref = np.ones(o.n, bool) if thr == 0.0 else mx > thr
        assert np.array_equal(gm[b].astype(bool), ref), f"block {b}"


def test_points_path_and_grid_agree():
    m, o = _pair(os.path.join(GOLDEN, "o2.fchk.gz"))
    grid = m.grid_around(1.0, 0.7)
    pts = grid.points()
    props = [K.density(P.Density), K.density(P.Gradient), K.density(P.Elf)]
    a, _ = K.Evaluator(m).evaluate_grid(grid, props)
    b, _ = K.Evaluator(m).evaluate_points(pts, props)
    refs, _ = o.evaluate([(int(p.kind), 0, 0, 0) for p in props], points=pts)
    _compare(b, refs, 1e-12, props)
    _compare(a, [x for x in b], 1e-12, props)


def test_grid_path_densities_ao_p():
    """AO-P densities on a grid take the values-only path (src/density.cpp:366-444)."""
    m, o = _pair(os.path.join(GOLDEN, "o2.fchk.gz"))
    grid = m.grid_around(2.0, 0.4)
    props = [K.density(P.Density, c) for c in (D.Total, D.Alpha, D.Beta, D.Difference)]
    outs, used = K.Evaluator(m, backend=K.Backend.AO_P).evaluate_grid(grid, props)
    refs, _ = o.evaluate([(0, int(c), 0, 0) for c in (0, 1, 2, 3)], grid=(grid.origin, grid.steps, grid.counts),
                         backend=1)
    assert used == 1
    _compare(outs, refs, 1e-12, props)


def test_orbitals():
    m, o = _pair(os.path.join(GOLDEN, "o2.fchk.gz"))
    grid = m.grid_around(1.5, 0.5)
    props = [K.orbital(9), K.orbital(7, K.SpinChannel.Beta), K.orbital(3, K.SpinChannel.Alpha, P.OrbitalGradient),
             K.orbital(3, K.SpinChannel.Beta, P.OrbitalHessian)]
    outs, _ = K.Evaluator(m).evaluate_grid(grid, props)
    pts = grid.points()
    refs = []
    for p in props:
        ch = p.channel
        n = o.n
        c = (o.c_beta if (ch == 1 and o.c_beta is not None) else o.c_alpha)[(p.orbital_index - 1) * n:p.orbital_index * n]
        if p.kind == P.Orbital:
            refs.append((c @ o.ao_values(pts))[None])
        else:
            panels = o.ao_derivatives(pts, 2)
            sel = [1, 2, 3] if p.kind == P.OrbitalGradient else [4, 5, 6, 7, 8, 9]
            refs.append(np.stack([c @ panels[s] for s in sel]))
    _compare(outs, refs, 1e-12, props)
    # At arbitrary points every orbital property takes the orbital pass.
    outs2, _ = K.Evaluator(m).evaluate_points(pts, props)
    _compare(outs2, refs, 1e-12, props)


OE_ALL = [19, 20, 21, 22, 23, 26, 27, 28, 29]


@pytest.mark.parametrize("name,kinds", [("acrolein.fchk.gz", OE_ALL), ("h2o_b3lyp_def2tzvp.fchk.gz", OE_ALL),
                                        ("o2.fchk.gz", [19, 20, 21, 22, 23])])
def test_orbital_energy_fields(name, kinds):
    # ALIE, LEA, LEAE, chi, eta and the orbital-weighted Fukui functions
    # against the oracle's restatement, at box points (nuclei included), with
    # ragged blocks, and on a grid.
    m, o = _pair(os.path.join(GOLDEN, name))
    props = [K.density(k) for k in kinds]
    pts = _box_points(o.atom_xyz.reshape(-1, 3), 3000, 5)
    refs = O.orbital_energy_fields(o, pts, kinds)
    for bs in (128, 37):
        outs, _ = K.Evaluator(m, block_size=bs).evaluate_points(pts, props)
        _compare(outs, [r[None] for r in refs], 1e-12, props)
    grid = m.grid_around(2.0, 0.3)
    outs, _ = K.Evaluator(m).evaluate_grid(grid, props)
    refs = O.orbital_energy_fields(o, grid.points(), kinds)
    _compare(outs, [r[None] for r in refs], 1e-12, props)


def test_orbital_energy_fields_with_density_and_delta():
    # Mixed with point-path fields and orbitals in one request, a non-default
    # Fukui delta, and the mixed precision (the orbital-energy pass is FP64).
    m, o = _pair(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    pts = _box_points(o.atom_xyz.reshape(-1, 3), 1500, 9)
    props = [K.density(P.Density), K.density(P.OrbitalWeightedFukuiPlus), K.density(P.AverageLocalIonizationEnergy),
             K.orbital(15), K.density(P.OrbitalWeightedDualDescriptor)]
    refs = O.orbital_energy_fields(o, pts, [26, 19, 29], fukui_delta=0.05)
    for prec in (K.Precision.FP64, K.Precision.Mixed):
        outs, _ = K.Evaluator(m, fukui_delta=0.05, precision=prec).evaluate_points(pts, props)
        _compare([outs[1], outs[2], outs[4]], [r[None] for r in refs], 1e-12, [props[1], props[2], props[4]])
        alone, _ = K.Evaluator(m).evaluate_points(pts, [K.density(P.Density)])
        if prec == K.Precision.FP64:
            assert np.array_equal(outs[0], alone[0])


@pytest.mark.parametrize("key,kind,abs_", [("acrolein_alie", 19, 0.0), ("o2_lea", 20, 0.0), ("o2_leae", 21, 1e-10),
                                           ("acrolein_local_hardness", 23, 0.0)])
def test_orbital_energy_multiwfn_cubes_on_gpu(key, kind, abs_):
    g = np.load(os.path.join(GOLDEN, f"multiwfn_{key}.npz"))
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, str(g["fchk"])))
    outs, _ = K.Evaluator(m).evaluate_points(golden_points(g), [K.density(kind)])
    v, ref = outs[0][0], g["values"]
    assert np.max(np.abs(v - ref) / (2e-5 * np.abs(ref) + abs_ + 1e-300)) <= 1.0


def test_golden_gaussian_cubes_on_gpu():
    for key, comp in [("o2_density", 0), ("o2_spin", 3), ("acrolein_density", 0)]:
        g = np.load(os.path.join(GOLDEN, f"gaussian_{key}.npz"))
        m = K.Molecule.from_fchk(os.path.join(GOLDEN, str(g["fchk"])))
        outs, _ = K.Evaluator(m, backend=K.Backend.AO_P).evaluate_points(golden_points(g), [K.density(P.Density, comp)])
        v, ref = outs[0][0], g["values"]
        assert np.max(np.abs(v - ref)) <= 2e-3
        assert np.abs(v - ref).sum() / np.abs(ref).sum() <= 1e-5


def test_golden_multiwfn_on_gpu():
    for key, kind, comp, rel, abs_ in [("h2o_elf", 6, 0, 2e-5, 0.0), ("h2o_rdg", 7, 0, 2e-5, 0.0),
                                       ("h2o_sign_lambda2_rho", 8, 0, 2e-5, 0.0), ("o2_elf", 6, 0, 2e-5, 0.0),
                                       ("o2_lol", 10, 0, 2e-5, 0.0)]:
        g = np.load(os.path.join(GOLDEN, f"multiwfn_{key}.npz"))
        m = K.Molecule.from_fchk(os.path.join(GOLDEN, str(g["fchk"])))
        outs, _ = K.Evaluator(m).evaluate_points(golden_points(g), [K.Property(kind, comp)])
        ratio = np.abs(outs[0][0] - g["values"]) / (rel * np.abs(g["values"]) + abs_ + 1e-300)
        assert ratio.max() <= 1.0, key


def test_esp_exact_vs_oracle_and_multiwfn():
    for name in ["h2o_esp", "o2_esp"]:
        g = np.load(os.path.join(GOLDEN, f"multiwfn_{name}.npz"))
        path = os.path.join(GOLDEN, str(g["fchk"]))
        m, o = _pair(path)
        pts = golden_points(g)[:1500]
        outs, _ = K.Evaluator(m, potential_tolerance=0.0).evaluate_points(pts, [K.density(P.ElectrostaticPotential)])
        ref = O.OracleESP(o).evaluate(pts)
        assert scaled_error(outs[0][0], ref) <= 1e-12
        assert m.esp_pair_count() == O.OracleESP(o).pair_count
        d = np.min(np.linalg.norm(pts[:, None, :] - o.atom_xyz.reshape(-1, 3)[None], axis=2), axis=1)
        keep = d >= 1e-3
        ratio = np.abs(outs[0][0] - g["values"][:1500])[keep] / (2e-5 * np.abs(g["values"][:1500][keep]) + 1e-7)
        assert ratio.max() <= 1.0


@pytest.mark.parametrize("tol", [1e-8, 1e-6, 1e-4])
def test_esp_with_tolerance_within_bound(tol):
    # chem-kumo's potential_tolerance bounds the error at every point
    # (src/electrostatic_potential.cpp:501-521).  The device drops the pairs
    # whose bounds sum to at most half the tolerance and evaluates the others
    # exactly: against the exact oracle every value is within the tolerance,
    # and fewer pairs are evaluated as the tolerance grows.
    m, o = _pair(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    grid = m.grid_around(2.0, 0.6)
    esp = [K.density(P.ElectrostaticPotential)]
    got, _ = K.Evaluator(m, potential_tolerance=tol).evaluate_grid(grid, esp)
    ref = O.OracleESP(o).evaluate(grid.points())
    err = np.max(np.abs(got[0][0] - ref))
    used, total = m.esp_pairs_evaluated(tol), m.esp_pair_count()
    print("acrolein tolerance", tol, "max error", err, "pairs", used, "of", total)
    assert err <= tol
    assert used <= total and m.esp_pairs_evaluated(0.0) == total
    if tol >= 1e-6:
        assert used < total


def test_esp_mixed_vs_fp64(monkeypatch):
    # Mixed form of the potential: FP64 Boys values and nuclear term, FP32
    # Hermite recursion and compensated FP32 pair sums.  Against the FP64 form
    # (which the other tests hold to the oracle and to Multiwfn) on a grid
    # around acrolein and on water's and O2's Multiwfn points.  The Multiwfn
    # tolerance itself (2e-5 relative + 1e-7 absolute) is an FP64 one: where
    # the nuclear and electronic terms cancel, the FP32 rounding of the
    # electronic sum exceeds its absolute part.
    esp = [K.density(P.ElectrostaticPotential)]
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    grid = m.grid_around(2.0, 0.3)
    f64, _ = K.Evaluator(m).evaluate_grid(grid, esp)
    # Without the opt-in, Precision::Mixed evaluates the potential in FP64.
    monkeypatch.delenv("KUMO_ESP_MIXED", raising=False)
    same, _ = K.Evaluator(m, precision=K.Precision.Mixed).evaluate_grid(grid, esp)
    assert np.array_equal(same[0][0], f64[0][0])
    monkeypatch.setenv("KUMO_ESP_MIXED", "1")
    mix, _ = K.Evaluator(m, precision=K.Precision.Mixed).evaluate_grid(grid, esp)
    err = scaled_error(mix[0][0], f64[0][0])
    print("esp mixed acrolein grid scaled error", err)
    assert err <= 1e-7, err
    for name in ["h2o_esp", "o2_esp"]:
        g = np.load(os.path.join(GOLDEN, f"multiwfn_{name}.npz"))
        m = K.Molecule.from_fchk(os.path.join(GOLDEN, str(g["fchk"])))
        pts = golden_points(g)
        f64, _ = K.Evaluator(m).evaluate_points(pts, esp)
        mix, _ = K.Evaluator(m, precision=K.Precision.Mixed).evaluate_points(pts, esp)
        err = scaled_error(mix[0][0], f64[0][0])
        print("esp mixed", name, "scaled error", err)
        assert err <= 1e-7, (name, err)


@pytest.mark.parametrize("rows", [0, 16, 100000])
def test_mixed_exact_rows(monkeypatch, rows):
    # The mixed AO-MO contraction with the last `rows` rows of each block's K
    # order added in FP64 (0: every row on the tensor cores; 16: the default;
    # 100000: as many as the kernel's staging holds).
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    _, _, xyz = m.atoms()
    rng = np.random.default_rng(3)
    pts = np.concatenate([xyz + rng.normal(0.0, 0.05, xyz.shape),
                          rng.uniform(xyz.min(0) - 2.0, xyz.max(0) + 2.0, (4000, 3))])
    props = [K.density(k, c) for k, c in FIELDS]
    # The Hessian request runs the register-staged kernel (ten panels).
    hprops = [K.density(k) for k in (P.Density, P.Hessian, P.Laplacian)]
    f64, _ = K.Evaluator(m, backend=K.Backend.AO_MO).evaluate_points(pts, props)
    hf64, _ = K.Evaluator(m, backend=K.Backend.AO_MO).evaluate_points(pts, hprops)
    monkeypatch.setenv("KUMO_MIXED_EXACT_ROWS", str(rows))
    mixed = K.Evaluator(m, backend=K.Backend.AO_MO, precision=K.Precision.Mixed)
    mix, _ = mixed.evaluate_points(pts, props)
    hmix, _ = mixed.evaluate_points(pts, hprops)
    monkeypatch.delenv("KUMO_MIXED_EXACT_ROWS")
    for p, a, r in zip(hprops, hmix, hf64):
        assert np.all(np.isfinite(a)), p
        print("exact rows", rows, "ten panels", p, scaled_error(a, r))
        # FP32 exact rows in the ten-panel kernel (measured 7.6e-8, 1.3e-7
        # with none).
        assert scaled_error(a, r) <= 3e-7, (p, scaled_error(a, r))
    # FP64 exact rows: 16 hold rho, grad rho, lap rho and tau to 1.6e-9
    # scaled (measured), every row exact gives the FP64 path's values
    # (8.5e-16), none leaves the tensor cores' 1.6e-7.
    tol = {0: 5e-7, 16: 1e-8}.get(rows, 1e-12)
    for p, a, r in zip(props[:4], mix[:4], f64[:4]):
        assert np.all(np.isfinite(a)), p
        print("exact rows", rows, p, scaled_error(a, r))
        assert scaled_error(a, r) <= tol, (p, scaled_error(a, r))
    assert scaled_error(mix[4], f64[4]) <= 1e-5


def test_boys_device_matches_oracle():
    t = np.concatenate([np.linspace(0.0, 45.0, 2001), [1e-9, 39.999999, 40.0, 200.0, 1e4]])
    got = K.boys(t, 13)
    ref = np.stack([O.boys(x, 13) for x in t])
    assert np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)) <= 1e-14


def test_mixed_precision_water(water28):
    m = K.Molecule.from_fchk(water28)
    origin, steps, counts = synth.workload_grid("water_28", m.atoms()[2])
    grid = K.Grid(origin, steps, counts)
    props = [K.density(k, c) for k, c in FIELDS]
    f64, _ = K.Evaluator(m).evaluate_grid(grid, props)
    mix, _ = K.Evaluator(m, precision=K.Precision.Mixed).evaluate_grid(grid, props)
    for p, a, r in zip(props[:4], mix[:4], f64[:4]):
        print("water mixed", p, scaled_error(a, r))
        # Every row of this 28-AO molecule that reaches the exact-row floor
        # is taken in FP64 (measured 2e-15).
        assert scaled_error(a, r) <= 1e-10, (p, scaled_error(a, r))
    print("water mixed ELF", scaled_error(mix[4], f64[4]))
    assert scaled_error(mix[4], f64[4]) <= 1e-5


# Panel counts of the tensor-core contraction: 1 (values), 4 (+gradient),
# 5 (+Laplacian panel), 10 (+full Hessian); every density component.
MIXED_CASES = {
    "values": [P.Density],
    "gradient": [P.Density, P.Gradient, P.Tau, P.Elf],
    "laplacian": [P.Density, P.Gradient, P.Laplacian, P.Tau],
    "hessian": [P.Density, P.Hessian, P.Laplacian],
}


@pytest.mark.parametrize("case", list(MIXED_CASES))
@pytest.mark.parametrize("name", ["o2.fchk.gz", "acrolein.fchk.gz"])
def test_mixed_tensor_core_panels_and_components(name, case):
    m, o = _pair(os.path.join(GOLDEN, name))
    pts = _box_points(o.atom_xyz.reshape(-1, 3), 3000, 5)
    comps = [D.Total, D.Alpha, D.Beta, D.Difference] if name == "o2.fchk.gz" else [D.Total]
    props = [K.density(k, c) for k in MIXED_CASES[case] for c in comps
             if not (k == P.Elf and c == D.Difference)]  # ELF of the spin density is undefined
    f64, _ = K.Evaluator(m, backend=K.Backend.AO_MO).evaluate_points(pts, props)
    mix, used = K.Evaluator(m, backend=K.Backend.AO_MO, precision=K.Precision.Mixed).evaluate_points(pts, props)
    assert used == int(K.Backend.AO_MO)
    total = {p.kind: r for p, r in zip(props, f64) if p.component == D.Total}
    for p, a, r in zip(props, mix, f64):
        assert np.all(np.isfinite(a)), p
        # Measured at most 5.7e-8 (ELF 3.8e-7) over every panel count and
        # component.
        tol = 2e-6 if p.kind == P.Elf else 1e-7
        # alpha - beta cancels: its FP32-level error follows the channels'
        # scale, so it is measured against the total of the same kind.
        scale = max(1.0, np.abs(total[p.kind]).max()) if p.component == D.Difference else max(1.0, np.abs(r).max())
        err = np.abs(a - r).max() / scale
        print("panels", name, case, p, err)
        assert err <= tol, (p, err)


@pytest.mark.parametrize("case", ["gradient", "laplacian", "hessian"])
@pytest.mark.parametrize("name", ["o2.fchk.gz", "acrolein.fchk.gz"])
def test_mixed_tensor_core_ao_p(name, case):
    # The AO-P form (Y = P Phi on the tensor cores) against the FP64 AO-P path,
    # every density component.
    m, o = _pair(os.path.join(GOLDEN, name))
    pts = _box_points(o.atom_xyz.reshape(-1, 3), 2500, 6)
    comps = [D.Total, D.Alpha, D.Beta, D.Difference] if name == "o2.fchk.gz" else [D.Total]
    props = [K.density(k, c) for k in MIXED_CASES[case] for c in comps if not (k == P.Elf and c == D.Difference)]
    f64, used = K.Evaluator(m, backend=K.Backend.AO_P).evaluate_points(pts, props)
    mix, used_m = K.Evaluator(m, backend=K.Backend.AO_P, precision=K.Precision.Mixed).evaluate_points(pts, props)
    assert used == used_m == int(K.Backend.AO_P)
    total = {p.kind: r for p, r in zip(props, f64) if p.component == D.Total}
    for p, a, r in zip(props, mix, f64):
        assert np.all(np.isfinite(a)), p
        if p.kind == P.Elf:
            # Y = sum_j phi_j P_jk sums many cancelling density-matrix entries,
            # and D = tau - |grad rho|^2 / 8 rho of ELF cancels again: the
            # mixed AO-P form holds ELF to 1e-4 (the AO-MO form to 1e-5).
            print("aop", name, case, p, "abs", np.abs(a - r).max())
            assert np.abs(a - r).max() <= 1e-4, (p, np.abs(a - r).max())
            continue
        scale = max(1.0, np.abs(total[p.kind]).max()) if p.component == D.Difference else max(1.0, np.abs(r).max())
        print("aop", name, case, p, np.abs(a - r).max() / scale)
        # Measured at most 9.4e-8 (no exact rows in the AO-P form).
        assert np.abs(a - r).max() / scale <= 2e-7, (p, np.abs(a - r).max() / scale)


@pytest.mark.parametrize("extra", ["none", "hessian", "spin_gradient"])
def test_mixed_ao_p_grid_densities(extra):
    # On a grid the FP64 AO-P form takes each density on the blocked grid path;
    # the mixed form computes them in its tensor-core point pass.  A density
    # matrix whose components need no derivatives is contracted with the value
    # panel only, in the same pass as the other matrix: values only for both
    # ("none"), four panels of P_total with P_spin's values ("hessian"), and
    # four panels of P_spin with P_total's values ("spin_gradient").
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "o2.fchk.gz"))
    grid = m.grid_around(2.0, 0.25)
    props = [K.density(P.Density, c) for c in (D.Alpha, D.Beta, D.Difference, D.Total)]
    if extra == "hessian":
        props += [K.density(P.ReducedGradient), K.density(P.SignLambda2Density)]
    elif extra == "spin_gradient":
        props += [K.density(P.Gradient, D.Difference), K.density(P.Tau, D.Difference)]
    f64, used = K.Evaluator(m, backend=K.Backend.AO_P).evaluate_grid(grid, props)
    mix, used_m = K.Evaluator(m, backend=K.Backend.AO_P, precision=K.Precision.Mixed).evaluate_grid(grid, props)
    assert used == used_m == int(K.Backend.AO_P)
    rho = np.asarray(f64[3]).ravel()
    for p, a, r in zip(props, mix, f64):
        a, r = np.asarray(a).ravel(), np.asarray(r).ravel()
        assert np.all(np.isfinite(a)), p
        if p.kind == P.ReducedGradient:
            # RDG = |grad rho| / rho^(4/3): compared where rho > 1e-6.
            sel = rho > 1e-6
            print("gridaop", extra, p, "rdg", np.abs(a[sel] - r[sel]).max() / np.abs(r[sel]).max())
            assert np.abs(a[sel] - r[sel]).max() / np.abs(r[sel]).max() <= 5e-7, p  # measured 7.8e-8
            continue
        scale = max(1.0, np.abs(rho).max())
        print("gridaop", extra, p, np.abs(a - r).max() / scale)
        assert np.abs(a - r).max() / scale <= 2e-7, (p, np.abs(a - r).max() / scale)  # measured 9.4e-8


def test_mixed_tensor_core_ao_p_many_column_chunks(synth_cache):
    # 740 AOs: about six 128-column chunks of Y per block.
    m = K.Molecule.from_fchk(synth.workload_fchk("organic_740", synth_cache))
    pts = _box_points(m.atoms()[2], 1024, 4)
    props = [K.density(P.Density), K.density(P.Gradient), K.density(P.Laplacian), K.density(P.Tau)]
    f64, _ = K.Evaluator(m, backend=K.Backend.AO_P).evaluate_points(pts, props)
    mix, _ = K.Evaluator(m, backend=K.Backend.AO_P, precision=K.Precision.Mixed).evaluate_points(pts, props)
    for p, a, r in zip(props, mix, f64):
        print("chunks", p, scaled_error(a, r))
        assert scaled_error(a, r) <= 5e-7, (p, scaled_error(a, r))  # measured 2.4e-7


def test_mixed_tensor_core_several_mo_passes(synth_cache):
    # 76 occupied MOs: with the full Hessian (10 panels) a pass holds 48 MO
    # columns of tensor memory, so the contraction takes two passes.
    path = synth.workload_fchk("organic_740", synth_cache)
    m = K.Molecule.from_fchk(path)
    pts = _box_points(m.atoms()[2], 2048, 9)
    props = [K.density(P.Density), K.density(P.Hessian), K.density(P.Gradient), K.density(P.Laplacian)]
    f64, _ = K.Evaluator(m).evaluate_points(pts, props)
    mix, _ = K.Evaluator(m, precision=K.Precision.Mixed).evaluate_points(pts, props)
    for p, a, r in zip(props, mix, f64):
        print("mopasses", p, scaled_error(a, r))
        # FP32 exact rows in the ten-panel kernel: measured 4.6e-7.
        assert scaled_error(a, r) <= 1e-6, (p, scaled_error(a, r))


@pytest.mark.parametrize("precision", ["Mixed", "FP64"])
def test_streamed_result_copies_match(precision):
    # Page-locked outputs: each wave's finished points are copied while the
    # next wave runs (a small scratch budget forces many waves).  The values
    # equal those of pageable outputs (copied once at the end), for a
    # one-pass request and for a request with a second (ESP) pass.
    import torch
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    grid = m.grid_around(2.0, 0.3)
    prec = getattr(K.Precision, precision)
    for props in ([K.density(P.Density), K.density(P.Gradient), K.density(P.Tau), K.density(P.Elf)],
                  [K.density(P.Density), K.density(P.ElectrostaticPotential)]):
        os.environ["KUMO_SCRATCH_MB"] = "8"
        try:
            ev = K.Evaluator(m, precision=prec)
            paged, _ = ev.evaluate_grid(grid, props)
            pinned = [torch.empty((K.channels(p.kind), grid.npoints), dtype=torch.float64, pin_memory=True).numpy()
                      for p in props]
            for o in pinned:
                o.fill(np.nan)
            ev.evaluate_grid(grid, props, out=pinned)
            pts = grid.points()[::3]
            ppts = [torch.empty((K.channels(p.kind), len(pts)), dtype=torch.float64, pin_memory=True).numpy()
                    for p in props]
            ev.evaluate_points(pts, props, out=ppts)
            ref_pts, _ = ev.evaluate_points(pts, props)
        finally:
            del os.environ["KUMO_SCRATCH_MB"]
        whole, _ = K.Evaluator(m, precision=prec).evaluate_grid(grid, props)
        for a, b, c in zip(paged, pinned, whole):
            assert np.array_equal(a, b)
            assert np.array_equal(a, c)
        for a, b in zip(ppts, ref_pts):
            assert np.array_equal(a, b)


def test_host_api_writes_into_caller_arrays():
    # Host-output calls copy each property from the device straight into the
    # caller's arrays; page-locked arrays reused across calls give the same
    # values as fresh ones, for grids and for explicit points.
    import torch
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    grid = m.grid_around(2.0, 0.35)
    props = [K.density(P.Density), K.density(P.Gradient), K.density(P.Laplacian), K.density(P.Elf)]
    ev = K.Evaluator(m, precision=K.Precision.Mixed)
    fresh, _ = ev.evaluate_grid(grid, props)
    pinned = [torch.empty((K.channels(p.kind), grid.npoints), dtype=torch.float64, pin_memory=True).numpy()
              for p in props]
    for _ in range(2):
        for o in pinned:
            o.fill(np.nan)
        got, _ = ev.evaluate_grid(grid, props, out=pinned)
        assert all(g is o for g, o in zip(got, pinned))
        for a, b in zip(fresh, pinned):
            assert np.array_equal(a, b)
    pts = grid.points()[::7]
    ref, _ = K.Evaluator(m).evaluate_points(pts, props)
    out = [np.full((K.channels(p.kind), len(pts)), np.nan) for p in props]
    K.Evaluator(m).evaluate_points(pts, props, out=out)
    for a, b in zip(ref, out):
        assert np.array_equal(a, b)
    with pytest.raises(K.InvalidArgument):
        ev.evaluate_grid(grid, props, out=pinned[:2])


def test_device_api_matches_host():
    import torch
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "h2o_b3lyp_def2tzvp.fchk.gz"))
    grid = m.grid_around(2.0, 0.3)
    props = [K.density(P.Density), K.density(P.Gradient), K.density(P.Elf)]
    host, _ = K.Evaluator(m).evaluate_grid(grid, props)
    outs = [torch.zeros(K.channels(p.kind) * grid.npoints, dtype=torch.float64, device="cuda") for p in props]
    stream = torch.cuda.current_stream().cuda_stream
    K.Evaluator(m).evaluate_grid_device(grid, props, [o.data_ptr() for o in outs], stream)
    torch.cuda.synchronize()
    for h, d in zip(host, outs):
        assert np.array_equal(h.ravel(), d.cpu().numpy())


def test_repeatable():
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    grid = m.grid_around(2.0, 0.4)
    props = [K.density(P.Density), K.density(P.Laplacian), K.density(P.Elf)]
    a, _ = K.Evaluator(m).evaluate_grid(grid, props)
    b, _ = K.Evaluator(m).evaluate_grid(grid, props)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_fused_mixed_form_matches_two_kernel_form():
    # The opt-in fused mixed AO-MO kernel (AO rows built inside the
    # tensor-core kernel, KUMO_MIXED_FUSED=1) against the two-kernel form and
    # the oracle, at the mixed tolerance.
    m, o = _pair(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    pts = _box_points(o.atom_xyz.reshape(-1, 3), 4000, 21)
    props = [K.density(P.Density), K.density(P.Gradient), K.density(P.Laplacian), K.density(P.Tau)]
    base, _ = K.Evaluator(m, precision=K.Precision.Mixed).evaluate_points(pts, props)
    os.environ["KUMO_MIXED_FUSED"] = "1"
    try:
        fused, used = K.Evaluator(m, precision=K.Precision.Mixed).evaluate_points(pts, props)
    finally:
        del os.environ["KUMO_MIXED_FUSED"]
    ref, _ = K.Evaluator(m).evaluate_points(pts, props)
    assert used == int(K.Backend.AO_MO)
    for p, a, b, r in zip(props, fused, base, ref):
        assert scaled_error(a, r) <= 1e-6, p
        assert scaled_error(a, b) <= 1e-6, p


@pytest.mark.parametrize("case", ["values", "gradient", "laplacian"])
@pytest.mark.parametrize("name", ["o2.fchk.gz", "acrolein.fchk.gz"])
def test_bulk_copy_contraction_equals_register_staged(name, case, monkeypatch):
    # The bulk-copy tensor-core contraction (rows fetched by tensor copies
    # into shared memory, the default) and the register-staged one
    # (KUMO_MIXED_BULK=0) split the same FP32 rows and accumulate the same
    # products in the same order when every row goes through the tensor cores
    # (KUMO_MIXED_EXACT_ROWS=0): the results agree bit for bit, and both hold
    # the mixed tolerance, as does the default bulk form with its exact rows.
    m, o = _pair(os.path.join(GOLDEN, name))
    pts = _box_points(o.atom_xyz.reshape(-1, 3), 5000, 33)
    comps = [D.Total, D.Alpha, D.Beta] if name == "o2.fchk.gz" else [D.Total]
    props = [K.density(k, c) for k in MIXED_CASES[case] for c in comps]
    default, _ = K.Evaluator(m, precision=K.Precision.Mixed).evaluate_points(pts, props)
    monkeypatch.setenv("KUMO_MIXED_EXACT_ROWS", "0")
    bulk, _ = K.Evaluator(m, precision=K.Precision.Mixed).evaluate_points(pts, props)
    os.environ["KUMO_MIXED_BULK"] = "0"
    try:
        staged, _ = K.Evaluator(m, precision=K.Precision.Mixed).evaluate_points(pts, props)
    finally:
        del os.environ["KUMO_MIXED_BULK"]
    ref, _ = K.Evaluator(m).evaluate_points(pts, props)
    for p, a, b, r, d in zip(props, bulk, staged, ref, default):
        assert np.array_equal(a, b), p
        print("bulk", name, case, p, scaled_error(a, r), scaled_error(d, r))
        # Measured: every row on the tensor cores 1.9e-7 (ELF 6.8e-7); the
        # default exact rows 4e-10 (ELF 5.1e-7).
        assert scaled_error(a, r) <= (2e-6 if p.kind == P.Elf else 5e-7), p
        assert scaled_error(d, r) <= (2e-6 if p.kind == P.Elf else 1e-8), p


def test_sharded_grid_equals_whole_grid():
    # Two block ranges evaluated as points (as two ranks would) give the
    # one-call grid result bit for bit.
    from kumo_b200 import shard
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    grid = m.grid_around(2.0, 0.3)
    props = [K.density(P.Density), K.density(P.Gradient), K.density(P.Elf)]
    whole, _ = K.Evaluator(m).evaluate_grid(grid, props)
    parts = []
    for r in range(3):
        first, count = shard.block_range(grid.npoints, r, 3)
        pts = shard.grid_points(grid.origin, grid.steps, grid.counts, first, count)
        parts.append(K.Evaluator(m).evaluate_points(pts, props)[0])
    for i in range(len(props)):
        assert np.array_equal(np.concatenate([p[i] for p in parts], axis=1), whole[i])


@pytest.mark.parametrize("counts", [(37, 23, 11), (40, 41, 1), (300, 1, 1), (1, 1, 129)])
def test_mixed_grid_tiles_padding(monkeypatch, counts):
    # The mixed form evaluates grids as compact tiles of 128 points (shapes
    # chosen per grid: cubes, planes, lines); partial tiles at the edges are
    # padding.  Against the FP64 form and against the same form on runs of
    # 128 points along k (KUMO_MIXED_TILES=0).  A line's tiles are as long as
    # runs of 128 points, so it gets the tolerance of linear blocks.
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    _, _, xyz = m.atoms()
    c = xyz.mean(axis=0)
    steps = np.diag([0.21, 0.19, 0.23])
    origin = c - 0.5 * np.array([(counts[a] - 1) * steps[a, a] for a in range(3)])
    grid = K.Grid(origin, steps, counts)
    props = [K.density(P.Density), K.density(P.Gradient), K.density(P.Laplacian), K.density(P.Tau),
             K.density(P.Elf)]
    f64, _ = K.Evaluator(m).evaluate_grid(grid, props)
    tiled, _ = K.Evaluator(m, precision=K.Precision.Mixed).evaluate_grid(grid, props)
    monkeypatch.setenv("KUMO_MIXED_TILES", "0")
    linear, _ = K.Evaluator(m, precision=K.Precision.Mixed).evaluate_grid(grid, props)
    dense = f64[0][0] > 1e-6  # ELF, a ratio, is compared where the density is not negligible
    compact = sorted(counts)[1] > 1  # tiles extend over at least two axes
    for p, t, l, r in zip(props, tiled, linear, f64):
        assert np.all(np.isfinite(t)), p
        if p.kind == P.Elf:
            t, l, r = t[:, dense], l[:, dense], r[:, dense]
        loose = 1e-5 if p.kind == P.Elf else 1e-6
        assert scaled_error(t, r) <= (1e-7 if compact else loose), (p, scaled_error(t, r))
        assert scaled_error(l, r) <= loose, (p, scaled_error(l, r))


def _field_errors(a, r, rho, positive):
    d = np.abs(a - r)
    out = {"scaled": float(d.max() / max(1.0, np.abs(r).max())),
           "pointwise": float((d / np.maximum(1.0, np.maximum(np.abs(a), np.abs(r)))).max())}
    if positive:
        m = rho > 1e-6
        out["rel"] = float((d[:, m] / np.abs(r[:, m])).max())
    return out


def test_mixed_accuracy_organic740_subgrid(synth_cache):
    # The headline request on the central 48^3 points of the 740-AO
    # molecule's 128^3 grid (the molecule's interior and valence shells):
    # mixed form against FP64, per field, in the reference's scaled metric and
    # (rho, tau, ELF) as the plain relative error where rho > 1e-6.
    m = K.Molecule.from_fchk(synth.workload_fchk("organic_740", synth_cache))
    origin, steps, counts = synth.workload_grid("organic_740", m.atoms()[2])
    sub = K.Grid(origin + steps @ np.array([40.0, 40.0, 40.0]), steps, (48, 48, 48))
    props = [K.density(P.Density), K.density(P.Gradient), K.density(P.Laplacian), K.density(P.Tau),
             K.density(P.Elf)]
    f64, _ = K.Evaluator(m).evaluate_grid(sub, props)
    mix, _ = K.Evaluator(m, precision=K.Precision.Mixed).evaluate_grid(sub, props)
    rho = f64[0][0]
    names = ["rho", "grad", "lap", "tau", "elf"]
    positive = [True, False, False, True, True]
    # Every field within 1e-7 in the reference's scaled metric (ELF, bounded
    # by 1, in absolute terms).  The plain relative error is printed: with
    # FP32 AO values it cannot reach 1e-7 at every point (the FP32 rounding
    # of exact AO values alone gives about 1e-7 on rho and 8e-7 on ELF).
    for name, a, r, pos in zip(names, mix, f64, positive):
        e = _field_errors(a, r, rho, pos)
        print("organic_740 48^3 mixed vs fp64", name, e)
        assert e["scaled"] <= 1e-7, (name, e)


def test_tile_autotuner_ranks_shapes_and_is_repeatable(monkeypatch):
    # Grids above 131,072 points: the mixed form times the compact tile
    # shapes on a probe sub-grid, keeps the ranking and evaluates with the
    # fastest; the result agrees with the default shape to the mixed
    # tolerance and repeats bit for bit.
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    _, _, xyz = m.atoms()
    n = 56
    grid = K.Grid(xyz.mean(axis=0) - 0.5 * 0.2 * (n - 1), np.eye(3) * 0.2, (n, n, n))
    props = [K.density(P.Density), K.density(P.Gradient), K.density(P.Laplacian), K.density(P.Tau)]
    ev = K.Evaluator(m, precision=K.Precision.Mixed)
    a, _ = ev.evaluate_grid(grid, props)
    report = K.tile_tuning_report()
    print(report)
    line = [l for l in report.splitlines() if "|5|" in l]
    assert line and len(line[-1].split()) >= 3  # key and at least two timed shapes
    b, _ = ev.evaluate_grid(grid, props)
    monkeypatch.setenv("KUMO_TILE_AUTOTUNE", "0")
    c, _ = ev.evaluate_grid(grid, props)
    f64, _ = K.Evaluator(m).evaluate_grid(grid, props)
    for x, y, z, r in zip(a, b, c, f64):
        assert np.array_equal(x, y)
        assert scaled_error(x, r) <= 1e-7 and scaled_error(z, r) <= 1e-7
