"""CPU model of the parallel cyclic Jacobi eigensolver of the Rayleigh-Ritz
kernel (k_small_eig, csrc/tof_lobpcg.cu): the same round-robin schedule, the
same rotation formula, stopping rule (relative criterion kJacTol, absolute
floor kJacAbs * ||A||_F, tested on every kJacTestEvery-th round) and four-term
element update.  Checks that the
schedule meets every pair exactly once per sweep for every basis size, that
each round keeps the matrix exactly symmetric, and that the eigenpairs match
LAPACK's on general, strongly graded and nearly singular (the SVQB path)
symmetric matrices."""
import numpy as np
import pytest

TOL, ABS = 1e-14, 1e-15
TEST_EVERY = 4       # the stopping test reads every fourth round's input


def schedule(K):
    """Pairs (p, q) of each round for K indices (padded to even NP)."""
    NP = K + (K & 1)
    M = NP - 1
    rounds = []
    for r in range(M):
        pairs = []
        for k in range(NP // 2):
            p = 0 if k == 0 else (r + k) % M + 1
            q = r + 1 if k == 0 else (r - k + M) % M + 1
            pairs.append((min(p, q), max(p, q)))
        rounds.append(pairs)
    return rounds


def live(apq, app, aqq, floor2):
    a2 = apq * apq
    return a2 > TOL * TOL * abs(app * aqq) and a2 > floor2


def jacobi(A0):
    K = A0.shape[0]
    A, V = A0.copy(), np.eye(K)
    floor2 = ABS * ABS * np.sum(A * A)
    rounds = schedule(K)
    for it in range(40 * len(rounds)):
        al, be, mt = np.ones(K + 1), np.zeros(K + 1), np.arange(K + 1)
        for p, q in rounds[it % len(rounds)]:
            if q < K and live(A[p, q], A[p, p], A[q, q], floor2):
                d, e = A[q, q] - A[p, p], 2.0 * A[p, q]
                r = np.sqrt(d * d + e * e)
                iw = 1.0 / np.sqrt(2.0 * r * (r + abs(d)))
                c, s = (r + abs(d)) * iw, (e if d >= 0 else -e) * iw
                al[p], be[p], mt[p] = c, -s, q
                al[q], be[q], mt[q] = c, s, p
        if it % TEST_EVERY == 0 and not any(live(A[i, j], A[i, i], A[j, j], floor2)
                                            for i in range(K) for j in range(K) if i != j):
            return np.diag(A).copy(), V
        An, Vn = np.empty_like(A), np.empty_like(V)
        for i in range(K):
            for j in range(K):
                mi, mj = mt[i], mt[j]
                if mi == j and mi != i:
                    An[i, j] = 0.0
                else:
                    t1 = (al[i] * al[j]) * A[i, j]
                    t2 = (al[i] * be[j]) * A[i, mj]
                    t3 = (be[i] * al[j]) * A[mi, j]
                    t4 = (be[i] * be[j]) * A[mi, mj]
                    An[i, j] = (t1 + (t2 + t3)) + t4
                Vn[i, j] = be[j] * V[i, mj] + al[j] * V[i, j]
        assert np.array_equal(An, An.T)
        A, V = An, Vn
    raise AssertionError("no convergence")


@pytest.mark.parametrize("K", range(1, 25))
def test_schedule_meets_every_pair_once_per_sweep(K):
    rounds = schedule(K)
    NP = K + (K & 1)
    seen = [pq for pairs in rounds for pq in pairs]
    assert len(seen) == len(set(seen)) == NP * (NP - 1) // 2
    for pairs in rounds:
        idx = [x for pq in pairs for x in pq]
        assert sorted(idx) == list(range(NP))


@pytest.mark.parametrize("K,kind", [(24, "general"), (23, "graded"), (14, "graded"), (17, "near_singular"), (2, "general")])
def test_eigenpairs_match_lapack(K, kind):
    rng = np.random.default_rng(K)
    Q, _ = np.linalg.qr(rng.standard_normal((K, K)))
    if kind == "general":
        lam = rng.uniform(0.1, 10.0, K)
    elif kind == "graded":
        lam = np.logspace(-6, 0, K)
    else:
        lam = np.concatenate([rng.uniform(0.5, 2.0, K - 3), [1e-17, 0.0, 1e-13]])
    A = (Q * lam) @ Q.T
    A = 0.5 * (A + A.T)
    d, V = jacobi(A)
    w = np.linalg.eigvalsh(A)
    scale = np.linalg.norm(A)
    assert np.max(np.abs(np.sort(d) - w)) <= 1e-13 * scale
    assert np.linalg.norm(V.T @ V - np.eye(K)) <= 1e-13 * K
    assert np.linalg.norm(A @ V - V * d) <= 1e-13 * scale * K
