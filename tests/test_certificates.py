"""The CPU checker of infeasibility certificates (oracle/certificates.py).

Pinned on LPs whose infeasibility (or feasibility) is known by construction:
a certificate that proves a feasible LP infeasible would be a false proof,
so weak duality is checked on feasible LPs with random rays (the margin is
never positive), and known rays of infeasible LPs are accepted.
"""
from __future__ import annotations

import numpy as np

import mcpdlp
from certificates import check_certificate, dual_ray_margin, row_activity_ray
from mcpdlp import generators

INF = float("inf")


def two_rows_infeasible():
    # x1 + x2 = 1 and x1 + x2 = 3, 0 <= x <= 10: each row alone is feasible
    return mcpdlp.from_triplets(2, 2, [0, 0, 1, 1], [0, 1, 0, 1], [1.0, 1.0, 1.0, 1.0],
                                objective=[1.0, 1.0], var_lower=[0.0, 0.0], var_upper=[10.0, 10.0],
                                row_lower=[1.0, 3.0], row_upper=[1.0, 3.0])


def test_known_ray_of_two_rows_is_accepted():
    m = two_rows_infeasible()
    # y = (1, -1): g = 0, L = 0, U = 1*1 + (-1)*3 = -2  ->  L - U = 2 > 0
    assert dual_ray_margin(m, [1.0, -1.0]) == 2
    assert check_certificate(m, "dual_ray", -1, np.array([1.0, -1.0]))
    assert not check_certificate(m, "dual_ray", -1, np.array([-1.0, 1.0]))


def test_weak_duality_on_feasible_lps():
    rng = np.random.default_rng(0)
    for seed in range(3):
        m = generators.random_lp(seed + 1, 40, 120, 6)
        for _ in range(20):
            y = rng.normal(size=m.num_rows) * 10.0 ** rng.uniform(-3, 3)
            mg = dual_ray_margin(m, y)
            assert mg is None or mg <= 0


def test_row_activity_and_crossed_bounds():
    bad = mcpdlp.from_triplets(1, 2, [0, 0], [0, 1], [1.0, 1.0], objective=[1.0, 1.0],
                               var_lower=[0.0, 0.0], var_upper=[2.0, 2.0], row_lower=[5.0],
                               row_upper=[5.0])
    assert row_activity_ray(bad, 0) is not None
    assert check_certificate(bad, "row_activity", 0, None)
    good = generators.random_lp(1, 40, 120, 6)
    assert not any(check_certificate(good, "row_activity", i, None) for i in range(good.num_rows))
    crossed = good.copy()
    crossed.var_lower = crossed.var_lower.copy()
    crossed.var_lower[7] = crossed.var_upper[7] + 1.0
    assert check_certificate(crossed, "crossed_bounds", 7, None)
    assert not check_certificate(crossed, "crossed_bounds", 6, None)


def test_infinite_bounds_void_a_ray():
    # x free: any nonzero g_j meets an infinite bound
    m = mcpdlp.from_triplets(2, 1, [0, 1], [0, 0], [1.0, 1.0], objective=[0.0], var_lower=[-INF],
                             var_upper=[INF], row_lower=[1.0, 3.0], row_upper=[1.0, 3.0])
    assert dual_ray_margin(m, [1.0, 0.0]) is None
    # rows x = 1 and x = 3 on a free x: the ray (1, -1) has g = 0 -> margin 2
    assert dual_ray_margin(m, [1.0, -1.0]) == 2
