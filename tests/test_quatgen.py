"""The product's orientation generator against the reference's quat_gen."""
import os

import numpy as np
import pytest

from common import GOLDEN
from dragonfly_b200.quatgen import quat_gen


@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_quat_gen_matches_reference_golden(n):
    g = np.load(os.path.join(GOLDEN, "quat_gen.npz"))["num_div_%d" % n]
    q = quat_gen(n)
    np.testing.assert_array_equal(q, g)


@pytest.mark.parametrize("n", [1, 2, 5, 10])
def test_quat_gen_invariants(n):
    """Known answers of quaternion.c: count 10 (5 n^3 + n) (quaternion.c:325),
    unit norm, weights summing to one (quaternion.c:835-839), q and -q never
    both present."""
    q = quat_gen(n)
    assert q.shape == (10 * (5 * n ** 3 + n), 5)
    np.testing.assert_allclose(np.linalg.norm(q[:, :4], axis=1), 1., rtol=0, atol=1e-14)
    assert abs(q[:, 4].sum() - 1.) < 1e-12
    assert (q[:, 4] > 0).all()
    # q and -q (or a repeat) would coincide after fixing the sign of the
    # first non-zero component
    c = q[:, :4].copy()
    first = np.argmax(np.abs(c) > 1e-12, axis=1)
    c *= np.sign(c[np.arange(len(c)), first])[:, None]
    assert np.unique(np.round(c, 9), axis=0).shape[0] == len(c)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref",
                                                    "libdragonfly_ref.so")),
                    reason="reference sources not compiled here")
@pytest.mark.parametrize("n", [5, 6, 10, 12])
def test_quat_gen_matches_live_reference(n):
    from oracle.oracle import quat_gen_reference
    np.testing.assert_array_equal(quat_gen(n), quat_gen_reference(n))
