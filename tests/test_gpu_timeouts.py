"""Failure reporting of the tensor-core pipelines without a GPU fault: every
mbarrier wait of the mixed contractions is bounded, and a wait that runs out
sets a device status word, stores NaN for its block's points, drains its own
MMAs and copies (with the full one-second limit) and frees tensor memory.
KUMO_PIPELINE_WAIT_NS shortens the pipeline waits to 1 ns, so that they run
out; the host-output call must then raise, the outputs of the failed blocks
must be NaN (the others exact), and the next evaluation with the normal limit
must give the normal result (the context stays usable and the status word is
cleared)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

import kumo_b200 as K
from kumo_b200 import synth

pytestmark = pytest.mark.gpu

P = K.PropertyKind

# The register-staged and AO-P kernels wait only on their own MMAs, which on
# a small molecule are done before the wait starts: those cases use the
# 740-AO molecule, whose longer K loops keep waits pending.
CASES = {
    "bulk_gradient": (K.Backend.AO_MO, [P.Density, P.Gradient, P.Tau, P.Elf], "acrolein"),
    "bulk_laplacian": (K.Backend.AO_MO, [P.Density, P.Gradient, P.Laplacian, P.Tau], "acrolein"),
    "register_staged_hessian": (K.Backend.AO_MO, [P.Density, P.Hessian], "organic_740"),
    "ao_p": (K.Backend.AO_P, [P.Density, P.Gradient, P.Laplacian], "organic_740"),
}


@pytest.mark.parametrize("case", list(CASES))
def test_pipeline_wait_timeout_is_reported_and_recovers(monkeypatch, synth_cache, case):
    backend, kinds, name = CASES[case]
    path = (os.path.join(GOLDEN, "acrolein.fchk.gz") if name == "acrolein"
            else synth.workload_fchk(name, synth_cache))
    m = K.Molecule.from_fchk(path)
    _, _, xyz = m.atoms()
    rng = np.random.default_rng(17)
    pts = rng.uniform(xyz.min(0) - 2.0, xyz.max(0) + 2.0, (3000, 3))
    props = [K.density(k) for k in kinds]
    ev = K.Evaluator(m, backend=backend, precision=K.Precision.Mixed)
    good, _ = ev.evaluate_points(pts, props)
    monkeypatch.setenv("KUMO_PIPELINE_WAIT_NS", "1")
    out = [np.full((K.channels(p.kind), len(pts)), -7.0) for p in props]
    with pytest.raises(K.KumoError, match="pipeline wait timed out"):
        ev.evaluate_points(pts, props, out=out)
    # Failed blocks hold NaN densities (and fields of them, such as ELF, that
    # treat a non-positive density as none); blocks whose waits never blocked
    # hold the result.
    nan_cols = np.isnan(out[0][0])
    assert nan_cols.any()
    for p, o, g in zip(props, out, good):
        if p.kind != P.Elf:
            assert np.array_equal(np.isnan(o).any(axis=0), nan_cols)
        assert np.array_equal(o[:, ~nan_cols], g[:, ~nan_cols])
    monkeypatch.delenv("KUMO_PIPELINE_WAIT_NS")
    again, _ = ev.evaluate_points(pts, props)
    for a, g in zip(again, good):
        assert np.array_equal(a, g)
    f64, _ = K.Evaluator(m, backend=backend).evaluate_points(pts, props)
    assert all(np.all(np.isfinite(x)) for x in f64)
