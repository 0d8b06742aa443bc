"""FP64 parity of the CUDA path with the oracle on the benchmark workloads
themselves (not scaled-down stand-ins): the 740-AO organic molecule on its
128^3 grid, the 3,700-AO unrestricted triplet on its 192^3 grid at screening
threshold 1e-10, and the exact potential of the 1,260-AO molecule on its 96^3
cube and its rho = 0.001 isosurface.  The oracle evaluates evenly spaced
128-point blocks of each grid (block structure kept, so the screening masks
are the same), at the tolerances of the other parity tests: 1e-12 in the
scaled metric max|gpu - ref| / max(1, max|ref|) of
tests/density_screening_test.cpp:137-150 (chem-kumo), ratio fields 1e-9
where rho > 1e-6, masks bit-exact."""
import numpy as np
import pytest

from conftest import scaled_error

import kumo_b200 as K
from kumo_b200 import synth
import oracle as O

pytestmark = pytest.mark.gpu

P = K.PropertyKind
D = K.DensityComponent


def _block_ids(npoints, nblocks):
    nb = (npoints + 127) // 128
    return np.unique(np.linspace(0, nb - 1, nblocks).astype(int))


def _take_blocks(values, ids, npoints):
    """Columns of the given 128-point blocks of a (channels, npoints) array."""
    cols = np.concatenate([np.arange(b * 128, min((b + 1) * 128, npoints)) for b in ids])
    return values[:, cols]


def test_organic740_fp64_grid_vs_oracle(synth_cache):
    # The headline workload's request (rho, grad rho, lap rho, tau, ELF) on the
    # whole 128^3 grid in FP64; 48 evenly spaced blocks against the oracle.
    path = synth.workload_fchk("organic_740", synth_cache)
    m = K.Molecule.from_fchk(path)
    o = O.OracleMolecule.from_fchk(path)
    origin, steps, counts = synth.workload_grid("organic_740", o.atom_xyz.reshape(-1, 3))
    grid = K.Grid(origin, steps, counts)
    props = [K.density(P.Density), K.density(P.Gradient), K.density(P.Laplacian), K.density(P.Tau),
             K.density(P.Elf)]
    outs, used = K.Evaluator(m).evaluate_grid(grid, props)
    ids = _block_ids(grid.npoints, 48)
    pts = np.concatenate([grid.points()[b * 128:(b + 1) * 128] for b in ids])
    refs, rused = o.evaluate([(int(p.kind), 0, 0, 0) for p in props], points=pts)
    assert used == rused == int(K.Backend.AO_MO)
    rho = refs[0][0]
    for p, a, r in zip(props, outs, refs):
        a = _take_blocks(a, ids, grid.npoints)
        err = scaled_error(a, r)
        print("organic_740 fp64", P(p.kind).name, "scaled error", err)
        if p.kind == P.Elf:
            dense = rho > 1e-6
            assert scaled_error(a[:, dense], r[:, dense]) <= 1e-12, err
            assert err <= 1e-10
        else:
            assert err <= 1e-12, (p, err)
    # Screening masks of those blocks (AO order 2, threshold 1e-12), bit-exact.
    masks = m.screening_masks(grid, 128, 2, 1e-12)
    flips = 0
    for b in ids:
        blk = grid.points()[b * 128:(b + 1) * 128]
        ref = np.abs(o.ao_derivatives(blk, 2)).max(axis=(0, 2)) > 1e-12
        flips += int(np.count_nonzero(masks[b].astype(bool) != ref))
    print("organic_740 screening mask flips over", len(ids), "blocks:", flips)
    assert flips == 0


TRIPLET = [(P.Density, D.Alpha), (P.Density, D.Beta), (P.Density, D.Difference), (P.Density, D.Total),
           (P.ReducedGradient, D.Total), (P.SignLambda2Density, D.Total)]


@pytest.mark.parametrize("backend", [K.Backend.AO_MO, K.Backend.AO_P])
def test_triplet3700_fp64_vs_oracle(synth_cache, backend):
    # The unrestricted 200-atom triplet (3,700 AOs, 381 alpha / 379 beta
    # electrons): alpha, beta and spin densities, RDG and sign(lambda2) rho
    # from the full AO Hessian, screening threshold 1e-10, on 32 evenly
    # spaced blocks of its 192^3 grid, both backends.
    path = synth.workload_fchk("triplet_3700", synth_cache)
    m = K.Molecule.from_fchk(path)
    o = O.OracleMolecule.from_fchk(path)
    assert o.n == 3700 and (o.nalpha, o.nbeta) == (381, 379)
    origin, steps, counts = synth.workload_grid("triplet_3700", o.atom_xyz.reshape(-1, 3))
    grid = K.Grid(origin, steps, counts)
    ids = _block_ids(grid.npoints, 32)
    pts = np.concatenate([grid.points()[b * 128:(b + 1) * 128] for b in ids])
    props = [K.density(k, c) for k, c in TRIPLET]
    outs, used = K.Evaluator(m, backend=backend, threshold=1e-10).evaluate_points(pts, props)
    refs, rused = o.evaluate([(int(p.kind), int(p.component), 0, 0) for p in props], points=pts,
                             backend=int(backend), threshold=1e-10)
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
            err = scaled_error(a, r)
            print("triplet_3700", backend.name, P(p.kind).name, D(p.component).name, "scaled error", err)
            assert err <= 1e-12, (p, err)


def test_esp1260_exact_vs_oracle(synth_cache):
    # Exact potential (tolerance 0) of the 1,260-AO molecule at 1,000 points
    # of its 96^3 cube and 1,000 vertices of its rho = 0.001 isosurface.
    path = synth.workload_fchk("esp_1260", synth_cache)
    m = K.Molecule.from_fchk(path)
    o = O.OracleMolecule.from_fchk(path)
    origin, steps, counts = synth.workload_grid("esp_1260", o.atom_xyz.reshape(-1, 3))
    cube = O.grid_points(origin, steps, counts)
    cube = cube[np.linspace(0, len(cube) - 1, 1000).astype(int)]
    surf = K.density_isosurface(m, 1e-3, 0.25).vertices
    surf = surf[np.linspace(0, len(surf) - 1, 1000).astype(int)]
    esp = O.OracleESP(o)
    assert m.esp_pair_count() == esp.pair_count
    # Each value sums about a million primitive-pair terms of both signs,
    # far larger than the result; the device (fixed-order partial sums per
    # pair chunk) and the oracle (left to right) round differently, so the
    # bound is 5e-11 here rather than the 1e-12 of the density fields
    # (measured: 5.9e-12 on the cube, 1.5e-11 on the surface).
    errs = {}
    for name, pts in (("cube", cube), ("surface", surf)):
        got, _ = K.Evaluator(m, potential_tolerance=0.0).evaluate_points(pts, [K.density(P.ElectrostaticPotential)])
        ref = esp.evaluate(pts)
        errs[name] = scaled_error(got[0][0], ref)
        print("esp_1260", name, "scaled error", errs[name])
    assert max(errs.values()) <= 5e-11, errs


@pytest.mark.parametrize("tol", [1e-8, 1e-6])
def test_esp1260_tolerance_within_bound(synth_cache, tol):
    # The potential with the tolerances of the ESP workload against the exact
    # one (tolerance 0, itself held to the oracle above) at 1,000 cube and
    # 1,000 isosurface points: every value within the tolerance.
    path = synth.workload_fchk("esp_1260", synth_cache)
    m = K.Molecule.from_fchk(path)
    _, _, xyz = m.atoms()
    origin, steps, counts = synth.workload_grid("esp_1260", xyz)
    cube = K.Grid(origin, steps, counts).points()
    cube = cube[np.linspace(0, len(cube) - 1, 1000).astype(int)]
    surf = K.density_isosurface(m, 1e-3, 0.25).vertices
    surf = surf[np.linspace(0, len(surf) - 1, 1000).astype(int)]
    prop = [K.density(P.ElectrostaticPotential)]
    for name, pts in (("cube", cube), ("surface", surf)):
        exact, _ = K.Evaluator(m, potential_tolerance=0.0).evaluate_points(pts, prop)
        got, _ = K.Evaluator(m, potential_tolerance=tol).evaluate_points(pts, prop)
        err = float(np.max(np.abs(got[0][0] - exact[0][0])))
        print("esp_1260", name, "tolerance", tol, "max error", err, "pairs", m.esp_pairs_evaluated(tol), "of",
              m.esp_pair_count())
        assert err <= tol, (name, err)
