"""The adjoint's CPU oracle (tests/golden/adjoint_c4.npz, made by make_adjoint_golden.py from
oracle/adjoint_ref on the reference's own transport).

The reference has no adjoint, so its oracle is pinned in two steps: the CPU restatement of
the transport loop that carries the scores reproduces the reference's hits bit for bit
(`check`), and its score-function estimate agrees with central finite differences with
common random numbers on the unmodified reference transport within 3 sigma."""
import numpy as np

from tests.helpers import golden


def test_restated_loop_is_the_reference():
    ref = golden("adjoint_c4.npz")
    assert int(ref["check_events"]) >= 10_000
    assert int(ref["check_mismatched"]) == 0


def test_reference_estimator_matches_reference_finite_differences():
    ref = golden("adjoint_c4.npz")
    for k in range(4):
        z = (ref["est_mean"][1 + k] - ref["fd_mean"][k]) / np.hypot(ref["est_se"][1 + k], ref["fd_se"][k])
        assert abs(z) < 3.0, (k, z)


def test_fixture_weights_are_the_loss_gradient():
    ref = golden("adjoint_c4.npz")
    n = float(ref["n"])
    np.testing.assert_allclose(ref["w"], 2.0 * (ref["hist0"] - ref["hist_target"]) / n, rtol=0, atol=0)
