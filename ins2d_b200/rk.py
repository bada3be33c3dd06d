"""Butcher tableaux of the explicit methods of unsteady/getRKmethod.m
(table data: A, b and c; c defaults to the row sums of A as in the
reference)."""
import numpy as np

_TABLES = {
    "FE11": ([[0]], [1], None),                                            # getRKmethod.m:20-24
    "SSP22": ([[0, 0], [1, 0]], [1 / 2, 1 / 2], None),                     # :26-29
    "SSP33": ([[0, 0, 0], [1, 0, 0], [1 / 4, 1 / 4, 0]], [1 / 6, 1 / 6, 2 / 3], None),  # :36-39
    "Wray3": ([[0, 0, 0], [8 / 15, 0, 0], [8 / 15 - 17 / 60, 5 / 12, 0]], [8 / 15 - 17 / 60, 0, 3 / 4],
              [0, 8 / 15, 8 / 15 - 17 / 60 + 5 / 12]),                      # :81-90
    "Heun33": ([[0, 0, 0], [1 / 3, 0, 0], [0, 2 / 3, 0]], [1 / 4, 0, 3 / 4], None),  # :296-299
    "RK33C2": ([[0, 0, 0], [2 / 3, 0, 0], [1 / 3, 1 / 3, 0]], [1 / 4, 0, 3 / 4], [0, 2 / 3, 2 / 3]),  # :301-305
    "RK33P2": ([[0, 0, 0], [1 / 3, 0, 0], [-1, 2, 0]], [0, 3 / 4, 1 / 4], [0, 1 / 3, 1]),  # :307-311
    "RK44": ([[0, 0, 0, 0], [1 / 2, 0, 0, 0], [0, 1 / 2, 0, 0], [0, 0, 1, 0]],
             [1 / 6, 1 / 3, 1 / 3, 1 / 6], None),                          # :313-316
    "RK44C2": ([[0, 0, 0, 0], [1 / 4, 0, 0, 0], [0, 1 / 2, 0, 0], [1, -2, 2, 0]],
               [1 / 6, 0, 2 / 3, 1 / 6], [0, 1 / 4, 1 / 2, 1]),            # :318-321
    "RK44C23": ([[0, 0, 0, 0], [1 / 2, 0, 0, 0], [1 / 4, 1 / 4, 0, 0], [0, -1, 2, 0]],
                [1 / 6, 0, 2 / 3, 1 / 6], [0, 1 / 2, 1 / 2, 1]),           # :323-327
    "RK44P2": ([[0, 0, 0, 0], [1, 0, 0, 0], [3 / 8, 1 / 8, 0, 0], [-1 / 8, -3 / 8, 3 / 2, 0]],
               [1 / 6, -1 / 18, 2 / 3, 2 / 9], [0, 1, 1 / 2, 1]),          # :329-333
}


def names():
    return sorted(_TABLES)


def getRKmethod(name):
    """[A, b, c] = getRKmethod(name) for the explicit methods above."""
    if name not in _TABLES:
        raise ValueError("RK method not available")
    A, b, c = _TABLES[name]
    A = np.array(A, dtype=float)
    b = np.array(b, dtype=float)
    c = A.sum(axis=1) if c is None else np.array(c, dtype=float)
    return A, b, c
