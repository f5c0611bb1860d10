"""The spectral pressure preconditioner's host-computed cyclic-reduction
tables (pvof_spectral_tables), on the CPU: replaying the reduction rounds
with them in numpy solves every wave number's tridiagonal system
-z_{j-1} + (b_j + dy^2 lambda_x) z_j - z_{j+1} = r_j (b_j = 2 inside, 1 at the
mirror walls) to 1e-12 relative of a direct solve; the mean mode (wave 0),
singular, gives the mean-free solution plus the right-hand side's mean."""
import ctypes as C
import math

import numpy as np
import pytest


def tables(N, M, idx2, idy2):
    from pvof.runtime import load
    L = load()
    L.pvof_spectral_tables.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.POINTER(C.c_double), C.c_longlong]
    L.pvof_spectral_tables.restype = C.c_longlong
    n = L.pvof_spectral_tables(N, M, idx2, idy2, None, 0)
    assert n > 0
    buf = np.zeros(n)
    assert L.pvof_spectral_tables(N, M, idx2, idy2, buf.ctypes.data_as(C.POINTER(C.c_double)), n) == n
    R = max(0, math.ceil(math.log2(M))) if M > 1 else 0
    assert n == (2 * R + 1) * (N // 2 + 1) * M
    return buf.reshape(2 * R + 1, N // 2 + 1, M), R


def replay(t, R, w, r):
    """the device's rounds: r_j -= k1 r_{j-s} + k2 r_{j+s}, then times 1 / b"""
    M = r.size
    r = r.copy()
    for st in range(R):
        s = 1 << st
        new = r.copy()
        for j in range(M):
            if j - s >= 0:
                new[j] -= r[j - s] * t[2 * st, w, j]
            if j + s < M:
                new[j] -= r[j + s] * t[2 * st + 1, w, j]
        r = new
    return r * t[2 * R, w]


def matrix(N, M, w, idx2, idy2):
    lam = (2.0 - 2.0 * math.cos(2.0 * math.pi * w / N)) * idx2 / idy2
    A = np.zeros((M, M))
    for j in range(M):
        A[j, j] = lam + (1.0 if j > 0 else 0.0) + (1.0 if j < M - 1 else 0.0)
        if j > 0:
            A[j, j - 1] = -1.0
        if j < M - 1:
            A[j, j + 1] = -1.0
    return A


@pytest.mark.parametrize("N,M,idx2,idy2", [(8, 5, 64.0, 64.0), (16, 16, 256.0, 64.0), (4, 33, 16.0, 100.0),
                                          (32, 1, 1024.0, 1024.0)])
def test_tables_solve_every_wave_number(N, M, idx2, idy2):
    t, R = tables(N, M, idx2, idy2)
    rng = np.random.default_rng(N * 1000 + M)
    for w in range(N // 2 + 1):
        r = rng.standard_normal(M)
        if w == 0:   # singular: the device pins row 0 of the mean-free right-hand side
            rm = r.mean()
            rr = r - rm
            rr[0] = 0.0
            x = replay(t, R, 0, rr)
            x = x - x.mean() + rm
            A = matrix(N, M, 0, idx2, idy2)
            # the mean-free part solves A x = r - mean(r); the mean is the right-hand side's
            assert np.abs(A @ (x - x.mean()) - (r - rm)).max() <= 1e-10 * max(1.0, np.abs(r).max())
            assert abs(x.mean() - rm) <= 1e-12 * max(1.0, abs(rm))
        else:
            x = replay(t, R, w, r)
            ref = np.linalg.solve(matrix(N, M, w, idx2, idy2), r)
            assert np.abs(x - ref).max() <= 1e-12 * np.abs(ref).max(), w


def test_invalid_sizes_are_refused():
    from pvof.runtime import load
    L = load()
    L.pvof_spectral_tables.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.POINTER(C.c_double), C.c_longlong]
    L.pvof_spectral_tables.restype = C.c_longlong
    assert L.pvof_spectral_tables(12, 8, 1.0, 1.0, None, 0) == -1
    assert L.pvof_spectral_tables(8, 0, 1.0, 1.0, None, 0) == -1
