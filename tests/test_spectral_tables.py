"""The spectral pressure preconditioner's host-computed table
(pvof_spectral_tables), on the CPU: replaying the device's partition-method
solve with it in numpy (chunk eliminations, the reduced system's Thomas
sweeps, back substitution) solves every wave number's tridiagonal system
-z_{j-1} + (b_j + dy^2 lambda_x) z_j - z_{j+1} = r_j (b_j = 2 inside, 1 at the
mirror walls) to a residual of 1e-10 of the right-hand side and within
1e-10 of a direct solve; the mean mode (wave 0), singular, gives the
mean-free solution plus the right-hand side's mean."""
import ctypes as C
import math

import numpy as np
import pytest


def chunks(M):
    """the partition of the M rows into P chunks (start, length), K the longest"""
    P = min(32, M // 2)
    base, rem = M // P, M % P
    return P, base + (1 if rem else 0), [(l * base + min(l, rem), base + (1 if l < rem else 0)) for l in range(P)]


def tables(N, M, idx2, idy2):
    from pvof.runtime import load
    L = load()
    L.pvof_spectral_tables.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.POINTER(C.c_double), C.c_longlong]
    L.pvof_spectral_tables.restype = C.c_longlong
    n = L.pvof_spectral_tables(N, M, idx2, idy2, None, 0)
    assert n > 0
    buf = np.zeros(n)
    assert L.pvof_spectral_tables(N, M, idx2, idy2, buf.ctypes.data_as(C.POINTER(C.c_double)), n) == n
    P, K, _ = chunks(M)
    assert n == (N // 2 + 1) * (2 * K + 4) * 32
    return buf.reshape(N // 2 + 1, 2 * K + 4, 32)


def replay(t, w, r):
    """the device's solve of one system with the wave number's table t[w]:
    per chunk the down sweep D_i = r_i (d_i + D_{i-1}) and the up sweep
    E_i = D_i + r_i E_{i+1}, the 2P chunk-end equations by Thomas with the
    table's pivots, then x_i = D_i - A_i x_first + r_i x_{i+1}"""
    M = r.size
    P, K, ch = chunks(M)
    T = t[w]
    col = r.astype(float).copy()
    rh, lo = np.zeros(2 * P), np.zeros(2 * P)
    for l, (s, L) in enumerate(ch):
        D = 0.0
        for i in range(1, L):
            D = T[i, l] * col[s + i] if i == 1 else T[i, l] * (col[s + i] + D)
            col[s + i] = D
        E = 0.0
        for i in range(L - 2, 0, -1):
            E = col[s + i] + T[i, l] * E
        rh[2 * l], lo[2 * l] = col[s] - T[0, l] * E, T[K, l]
        rh[2 * l + 1], lo[2 * l + 1] = D, T[K + L - 1, l]
    dp, prev = np.zeros(2 * P), 0.0
    for k in range(2 * P):
        prev = (rh[k] - lo[k] * prev) * T[2 * K + 2 * (k & 1), k // 2]
        dp[k] = prev
    x, nxt = np.zeros(2 * P), 0.0
    for k in range(2 * P - 1, -1, -1):
        nxt = dp[k] - T[2 * K + 2 * (k & 1) + 1, k // 2] * nxt
        x[k] = nxt
    for l, (s, L) in enumerate(ch):
        x0, xn = x[2 * l], x[2 * l + 1]
        col[s], col[s + L - 1] = x0, xn
        for i in range(L - 2, 0, -1):
            xn = col[s + i] - T[K + i, l] * x0 + T[i, l] * xn
            col[s + i] = xn
    return col


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
                                          (12, 40, 1.0, 1.0), (80, 160, 1.0, 1.0),
                                          (32, 2, 1024.0, 1024.0), (8, 3, 1.0, 1.0), (16, 1000, 1.0, 4.0),
                                          (8, 1023, 1.0, 1.0), (1024, 1024, 1.0, 1.0)])
def test_tables_solve_every_wave_number(N, M, idx2, idy2):
    t = tables(N, M, idx2, idy2)
    rng = np.random.default_rng(N * 1000 + M)
    waves = range(N // 2 + 1) if N <= 64 else sorted({0, 1, 2, 3, N // 4, N // 2 - 1, N // 2})
    for w in waves:
        r = rng.standard_normal(M)
        A = matrix(N, M, w, idx2, idy2)
        if w == 0:   # singular: the device pins row 0 of the mean-free right-hand side
            rm = r.mean()
            rr = r - rm
            rr[0] = 0.0
            x = replay(t, 0, rr)
            Ap = A.copy()
            Ap[0, :] = 0.0
            Ap[0, 0] = 1.0
            assert np.abs(Ap @ x - rr).max() <= 1e-10 * max(1.0, np.abs(rr).max())
            x = x - x.mean() + rm
            # the mean-free part solves A x = r - mean(r); the mean is the right-hand side's
            assert np.abs(A @ (x - x.mean()) - (r - rm)).max() <= 1e-10 * max(1.0, np.abs(r).max())
            assert abs(x.mean() - rm) <= 1e-12 * max(1.0, abs(rm))
        else:
            x = replay(t, w, r)
            ref = np.linalg.solve(A, r)
            assert np.abs(A @ x - r).max() <= 1e-10 * np.abs(r).max(), w
            assert np.abs(x - ref).max() <= 1e-10 * np.abs(ref).max(), w


def test_invalid_sizes_are_refused():
    from pvof.runtime import load
    L = load()
    L.pvof_spectral_tables.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.POINTER(C.c_double), C.c_longlong]
    L.pvof_spectral_tables.restype = C.c_longlong
    assert L.pvof_spectral_tables(14, 8, 1.0, 1.0, None, 0) == -1   # 7 x 2: not 2^a, 3 2^a or 5 2^a
    assert L.pvof_spectral_tables(15, 8, 1.0, 1.0, None, 0) == -1   # odd
    assert L.pvof_spectral_tables(8, 0, 1.0, 1.0, None, 0) == -1
    assert L.pvof_spectral_tables(8, 1, 1.0, 1.0, None, 0) == -1
