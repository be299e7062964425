"""The grouped LU scheme of the FP32 tensor-core path, restated in numpy and
checked against the one-panel-at-a-time blocked LU (CPU, no GPU).

lu_run (csrc/lu.cu) factors G = 2 or 4 consecutive 64-column panels per
trailing update: inside the group the LU is right-looking (each panel's
update reaches the group's remaining columns at once), while the columns past
the group receive the later panels' interchanges without the earlier panels'
updates.  Each panel's U rows past the group first take the deferred update
of the earlier panels of the group (their L read at this panel's rows through
the group's row maps), and the rest of the deferred work is one K = 64 G
update whose L is read through the same maps.  A keeps the factors of the
ordinary blocked LU (L in panel order, no interchanges left of a panel), so
the solves need no change.  This test restates that bookkeeping (the row
maps and their update new_map[dst] = old_map[src] over a panel's
interchanges) and checks that it reproduces the ordinary LU's pivots and
factors.
"""
import numpy as np
import pytest

NB = 64


def _panel_lu(A, k, w):
    """Partial pivoting (first row of largest |re|+|im|) of columns k..k+w-1
    on rows k.., interchanging whole rows of the panel columns; returns the
    list of (position, pivot position) pairs."""
    sw = []
    for j in range(k, k + w):
        p = j + int(np.argmax(np.abs(A[j:, j].real) + np.abs(A[j:, j].imag)))
        sw.append((j, p))
        if p != j:
            A[[j, p], k:k + w] = A[[p, j], k:k + w]
        A[j + 1:, j] /= A[j, j]
        A[j + 1:, j + 1:k + w] -= np.outer(A[j + 1:, j], A[j, j + 1:k + w])
    return sw


def _swap_rows(A, sw, cols):
    for j, p in sw:
        if p != j:
            A[[j, p], cols] = A[[p, j], cols]


def _blocked_lu(A0):
    A = A0.copy()
    n = A.shape[0]
    pivots = []
    for k in range(0, n, NB):
        sw = _panel_lu(A, k, NB)
        pivots.append(sw)
        c = slice(k + NB, n)
        _swap_rows(A, sw, c)
        L11 = np.tril(A[k:k + NB, k:k + NB], -1) + np.eye(NB)
        A[k:k + NB, c] = np.linalg.solve(L11, A[k:k + NB, c])
        A[k + NB:, c] -= A[k + NB:, k:k + NB] @ A[k:k + NB, c]
    return A, pivots


def _grouped_lu(A0, G):
    A = A0.copy()
    n = A.shape[0]
    pivots = []
    k = 0
    while k < n:
        g = min(G, (n - k) // NB)
        kG = k + NB * g
        maps = {}  # map j: position now -> position of that row after panel j
        for i in range(g):
            ki = k + NB * i
            sw = _panel_lu(A, ki, NB)
            pivots.append(sw)
            src = np.arange(n)  # after panel i, position x holds the row that was at src[x]
            for j, p in sw:
                src[[j, p]] = src[[p, j]]
            for j in maps:
                maps[j] = maps[j][src]
            if i < g - 1:
                maps[i] = np.arange(n)
            _swap_rows(A, sw, slice(ki + NB, n))
            L11 = np.tril(A[ki:ki + NB, ki:ki + NB], -1) + np.eye(NB)
            cg, cd = slice(ki + NB, kG), slice(kG, n)
            A[ki:ki + NB, cg] = np.linalg.solve(L11, A[ki:ki + NB, cg])
            B = A[ki:ki + NB, cd].copy()
            for j in range(i):  # the earlier panels' deferred update of this panel's rows
                kj = k + NB * j
                B -= A[maps[j][ki:ki + NB], kj:kj + NB] @ A[kj:kj + NB, cd]
            A[ki:ki + NB, cd] = np.linalg.solve(L11, B)
            if i < g - 1:  # the narrow update of the group's remaining columns
                A[ki + NB:, cg] -= A[ki + NB:, ki:ki + NB] @ A[ki:ki + NB, cg]
        if kG < n:  # one update of K = 64 g past the group, L through the row maps
            rows = [maps[j][kG:] if j < g - 1 else np.arange(kG, n) for j in range(g)]
            Lhat = np.hstack([A[rows[j], k + NB * j:k + NB * (j + 1)] for j in range(g)])
            Uhat = np.vstack([A[k + NB * j:k + NB * (j + 1), kG:] for j in range(g)])
            A[kG:, kG:] -= Lhat @ Uhat
        k = kG
    return A, pivots


@pytest.mark.parametrize("G", [2, 4])
def test_grouped_updates_reproduce_the_blocked_lu(G):
    rng = np.random.default_rng(1)
    n = 6 * NB
    A0 = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    R, piv_r = _blocked_lu(A0)
    Q, piv_q = _grouped_lu(A0, G)
    assert piv_q == piv_r
    assert np.abs(Q - R).max() <= 1e-10 * np.abs(R).max()
