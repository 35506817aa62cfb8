"""The differentiable form on the GPU: at the nominal parameters the forward image is the plain
renderer's, and the path-replay adjoint matches paired central finite differences (h = 1e-3) to
1e-3 relative on sky, emitter and albedo parameters of a small frame of the differentiation world."""

import numpy as np
import pytest

from lumenwright_b200 import adjoint as A

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem():
    from lumenwright_b200.native import Context
    c = Context(0)
    p = A.DiffProblem(c, width=96, height=54, spp=8)
    yield p
    c.close()


def test_forward_at_nominal_theta_is_the_render(problem):
    p = problem
    params, cache = p.frame(A.split(p.theta0).sky)
    want = p.ctx.render_hq(params, cache, p.spp).astype(np.float64)
    got = p.forward(p.theta0)
    assert np.all(np.abs(got - want) <= 1e-5 * np.maximum(np.abs(want), 1e-3))


def test_adjoint_matches_central_differences(problem):
    p = problem
    idx = p.check_indices(n=64, seed=3)
    loss, g, rows = A.check(p, idx)
    assert loss > 0.0
    fd = np.array([r["fd"] for r in rows])
    ad = np.array([r["adjoint"] for r in rows])
    assert np.count_nonzero(fd) >= 24
    # Relative 1e-3, with a floor for parameters whose derivative is tiny next to their class's.
    for lo, hi in ((0, A.N_ALBEDO), (A.N_ALBEDO, A.N_ALBEDO + A.GROUPS), (A.N_ALBEDO + A.GROUPS, A.N_THETA)):
        m = (idx >= lo) & (idx < hi)
        if not m.any():
            continue
        floor = 1e-6 * np.abs(fd[m]).max()
        bad = np.abs(ad[m] - fd[m]) > 1e-3 * np.maximum(np.abs(fd[m]), np.abs(ad[m])) + floor
        assert not bad.any(), [rows[i] for i in np.nonzero(m)[0][bad]]
