"""CPU check of infeasibility certificates -- TEST INFRASTRUCTURE ONLY.

The reference PDLP never returns infeasible_or_unbounded
(include/markov_cero/lp/first_order/pdlp.hpp:43 declares it; pdlp.cpp never
sets it), so there is no reference result to compare a certificate with.
This module checks each certificate on its own, in exact rational
arithmetic (fractions.Fraction of the binary doubles), against the LP

    row_lower <= A x <= row_upper,   var_lower <= x <= var_upper.

* crossed bounds: var_lower[j] > var_upper[j].
* dual ray y (the engine's sign convention, the reference's negated
  multiplier): with g = A^T y,
      L = sum_j (g_j > 0 ? g_j var_lower[j] : g_j var_upper[j])
      U = sum_i (y_i > 0 ? y_i row_upper[i] : y_i row_lower[i])
  every term finite and L > U.  For a feasible x, L <= g.x = y.(A x) <= U,
  so L > U proves infeasibility (Farkas' lemma for a box-constrained LP).
* row activity of row i: the ray -e_i (max activity below row_lower[i])
  or +e_i (min activity above row_upper[i]).

Only tests/ use it, as the checker of the engine's certificates.
"""
from __future__ import annotations

import math
from fractions import Fraction

import numpy as np


def _bound_term(coef: Fraction, lo: float, hi: float, use_lower_when_positive: bool):
    """coef * (lo if (coef > 0) == use_lower_when_positive else hi); None if
    that bound is infinite (the term is unbounded)."""
    if coef == 0:
        return Fraction(0)
    pick_lower = (coef > 0) == use_lower_when_positive
    b = lo if pick_lower else hi
    if math.isinf(b):
        return None
    return coef * Fraction(b)


def dual_ray_margin(model, y) -> Fraction | None:
    """L - U of the Farkas test for the ray y (exact); None if a term meets
    an infinite bound (then y proves nothing)."""
    y = np.asarray(y, dtype=np.float64)
    if y.shape != (model.num_rows,) or not np.all(np.isfinite(y)):
        return None
    yf = [Fraction(float(v)) for v in y]
    L = Fraction(0)
    for j in range(model.num_cols):
        g = Fraction(0)
        for p in range(int(model.col_start[j]), int(model.col_start[j + 1])):
            yi = yf[int(model.row_index[p])]
            if yi:
                g += Fraction(float(model.value[p])) * yi
        t = _bound_term(g, float(model.var_lower[j]), float(model.var_upper[j]), True)
        if t is None:
            return None
        L += t
    U = Fraction(0)
    for i in range(model.num_rows):
        t = _bound_term(yf[i], float(model.row_lower[i]), float(model.row_upper[i]), False)
        if t is None:
            return None
        U += t
    return L - U


def row_activity_ray(model, i: int):
    """The unit ray of a row-activity certificate on row i: whichever of
    -e_i, +e_i has a positive margin (None if neither)."""
    for sign in (-1.0, 1.0):
        y = np.zeros(model.num_rows)
        y[i] = sign
        mg = dual_ray_margin(model, y)
        if mg is not None and mg > 0:
            return y
    return None


def check_certificate(model, kind: str, index: int, dual) -> bool:
    """True iff the engine's certificate proves `model` infeasible."""
    if kind == "crossed_bounds":
        return 0 <= index < model.num_cols and model.var_lower[index] > model.var_upper[index]
    if kind == "row_activity":
        return 0 <= index < model.num_rows and row_activity_ray(model, index) is not None
    if kind == "dual_ray":
        mg = dual_ray_margin(model, dual)
        return mg is not None and mg > 0
    return False
