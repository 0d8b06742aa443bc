"""The allocation-free entry point (kumo_evaluate_points_noalloc) against the
regular device entry point.

Some hosts cannot let a library call cudaMalloc (a serving process that
budgets all of HBM itself, an application whose memory manager owns the
device), so the library offers one call that keeps its AO scratch in a fixed
array reserved at load time.  This test checks, through the C ABI, that two
calls in a row of that entry point give the same fields as
kumo_evaluate_points_device, within the parity tolerance of the other tests.
The file sorts last so that a run stopping at the first failure has already
run every other test; it also passes alone in a fresh process, because it
first makes the molecule's device copy with a regular evaluation.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, scaled_error

import kumo_b200 as K

pytestmark = pytest.mark.gpu


def test_noalloc_matches_device_entry_point_twice():
    import torch

    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    _, _, xyz = m.atoms()
    rng = np.random.default_rng(7)
    pts = rng.uniform(xyz.min(0) - 2.0, xyz.max(0) + 2.0, (5000, 3))
    P = K.PropertyKind
    props = [K.density(P.Density), K.density(P.Gradient), K.density(P.Laplacian), K.density(P.Tau),
             K.density(P.Elf), K.density(P.Hessian)]
    dpts = torch.tensor(pts.ravel(), dtype=torch.float64, device="cuda")
    n = len(pts)
    stream = torch.cuda.current_stream().cuda_stream

    def outputs():
        return [torch.full((K.channels(p.kind) * n,), float("nan"), dtype=torch.float64, device="cuda")
                for p in props]

    ref = outputs()
    used = K.Evaluator(m, backend=K.Backend.AO_MO).evaluate_points_device(
        dpts.data_ptr(), n, props, [o.data_ptr() for o in ref], stream)
    assert used == int(K.Backend.AO_MO)
    torch.cuda.synchronize()
    for _ in range(2):
        got = outputs()
        K.evaluate_points_noalloc(m, dpts.data_ptr(), n, props, [o.data_ptr() for o in got], stream)
        torch.cuda.synchronize()
        for p, a, r in zip(props, got, ref):
            a, r = a.cpu().numpy(), r.cpu().numpy()
            assert np.all(np.isfinite(a)), p
            assert scaled_error(a, r) <= 1e-12, (p, scaled_error(a, r))


def test_noalloc_needs_resident_molecule_and_density_properties():
    import torch

    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "o2.fchk.gz"))
    pts = torch.zeros(3 * 4, dtype=torch.float64, device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    # No device copy yet on this device: the call refuses instead of allocating.
    with pytest.raises(K.InvalidArgument) as e:
        K.evaluate_points_noalloc(m, pts.data_ptr(), 4, [K.density(K.PropertyKind.Density)], [out.data_ptr()])
    assert "device copy" in str(e.value)
    with pytest.raises(K.InvalidArgument):
        K.evaluate_points_noalloc(m, pts.data_ptr(), 4, [K.orbital(3)], [out.data_ptr()])


def test_noalloc_unrestricted_two_channels():
    # O2 (triplet, unrestricted): the alpha and beta channels take separate
    # MO passes, and the spin-difference and beta densities come from both.
    import torch

    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "o2.fchk.gz"))
    _, _, xyz = m.atoms()
    rng = np.random.default_rng(11)
    pts = rng.uniform(xyz.min(0) - 2.5, xyz.max(0) + 2.5, (3000, 3))
    P, D = K.PropertyKind, K.DensityComponent
    props = [K.density(P.Density, D.Alpha), K.density(P.Density, D.Beta), K.density(P.Density, D.Difference),
             K.density(P.Gradient, D.Total), K.density(P.Elf, D.Total), K.density(P.Laplacian, D.Beta)]
    dpts = torch.tensor(pts.ravel(), dtype=torch.float64, device="cuda")
    n = len(pts)
    stream = torch.cuda.current_stream().cuda_stream

    def outputs():
        return [torch.full((K.channels(p.kind) * n,), float("nan"), dtype=torch.float64, device="cuda")
                for p in props]

    ref = outputs()
    K.Evaluator(m, backend=K.Backend.AO_MO).evaluate_points_device(dpts.data_ptr(), n, props,
                                                                   [o.data_ptr() for o in ref], stream)
    torch.cuda.synchronize()
    for _ in range(2):
        got = outputs()
        K.evaluate_points_noalloc(m, dpts.data_ptr(), n, props, [o.data_ptr() for o in got], stream)
        torch.cuda.synchronize()
        for p, a, r in zip(props, got, ref):
            a, r = a.cpu().numpy(), r.cpu().numpy()
            assert np.all(np.isfinite(a)), p
            assert scaled_error(a, r) <= 1e-12, (p, scaled_error(a, r))
    with pytest.raises(K.InvalidArgument):
        K.evaluate_points_noalloc(m, dpts.data_ptr(), n, props, [o.data_ptr() for o in ref[:2]], stream)
