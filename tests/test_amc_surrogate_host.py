"""The host logic of the AMC continuation surrogate (zlatko_b200.amc_surrogate) on hand-made paths: the realised
value of the policy from the next exercise on, and the polynomial records it is compared with."""
from types import SimpleNamespace

import numpy as np

from zlatko_b200 import amc_surrogate as AS
from zlatko_b200 import spec as S


def _record(center, inv_scale, c):
    r = np.zeros(8, np.float32)
    r[2], r[3], r[4:8] = center, inv_scale, c
    return r


def test_poly_is_the_kernels_record_evaluation():
    rec = _record(0.01, 50.0, [1.0, -2.0, 0.5, 0.25])
    x = np.array([-0.02, 0.0, 0.03])
    z = (x - 0.01) * 50.0
    assert np.allclose(AS._poly(rec, x), 1.0 - 2.0 * z + 0.5 * z ** 2 + 0.25 * z ** 3)


def test_realised_value_of_the_policy_from_the_next_exercise():
    # Two exercises at dates 2 and 4 (times 1.0 and 2.0); three paths; continuation records on dates 0..3.
    trade = S.Bermudan(S.Swap(1e6, 0.02, True, [0.0, 1.0, 2.0, 3.0]), [1.0, 2.0])
    times = np.array([0.0, 0.5, 1.0, 1.5, 2.0, 2.5])
    x = np.zeros((6, 3))
    D = np.array([[1.0] * 3, [0.99] * 3, [0.98] * 3, [0.97] * 3, [0.96] * 3, [0.95] * 3])
    ev = np.array([[5.0, -1.0, 3.0],    # exercise 0: values; policy threshold 4 -> exercises path 0 only
                   [7.0, 6.0, 2.0]])    # exercise 1: threshold 2.5 -> paths 0 and 1 (path 2 at 2.0 < 2.5)
    decide = [_record(0.0, 1.0, [4.0, 0, 0, 0]), _record(0.0, 1.0, [2.5, 0, 0, 0])]
    cont = {j: _record(0.0, 1.0, [1.0, 0, 0, 0]) for j in range(4)}
    L = AS.BermudanLayout(trade, [2, 4], decide, cont, 0)
    a = AS.AmcPaths(SimpleNamespace(times=times), x, D, ev, [L])
    r = AS.realised(a, 0)
    # Dates 0, 1: next exercise is 0 (t = 1.0): path 0 exercises there, path 1 at exercise 1, path 2 never.
    for j in (0, 1):
        y, poly = r[j]
        assert np.allclose(y, [0.98 * 5.0 / D[j, 0], 0.96 * 6.0 / D[j, 1], 0.0])
        assert np.allclose(poly, 1.0)
    # Dates 2, 3 (t = 1.0, 1.5): the next exercise is 1 (t = 2.0), whatever happened at exercise 0.
    for j in (2, 3):
        y, _ = r[j]
        assert np.allclose(y, [0.96 * 7.0 / D[j, 0], 0.96 * 6.0 / D[j, 1], 0.0])
