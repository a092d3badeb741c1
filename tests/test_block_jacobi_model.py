"""A NumPy model of the device eigensolver (molgw_b200/csrc/eigh_jacobi.cu), step
for step: 32-row blocks visited in the round-robin order of Brent and Luk; per
block pair one sweep of the cyclic Jacobi method on the 64 x 64 subproblem
(round-robin rotations, Rutishauser's tangent t = 2 a_pq / (d + sign(d)
sqrt(d^2 + 4 a_pq^2)), d = a_qq - a_pp), skipped when every off-diagonal entry
is <= tau = 1e-14 ||A||_F and rotating down to tau/4 otherwise; the round's
rotation applied to A and V in one pass; sweeps until one skips every pair.

It pins the algorithm's properties on the CPU (convergence in a handful of
sweeps, eigenvalues to 1e-14 of the largest, orthogonal V); the GPU tests check
the kernels against the oracle through the contour-deformation and RI-metric
entry points."""
import numpy as np

KB, KS = 32, 64


def rr_pair(r, k, m):
    if k == 0:
        return 0, 1 + r
    return 1 + (r + k) % (m - 1), 1 + (r - k + (m - 1)) % (m - 1)


def inner_sweep(S, tau):
    Q = np.eye(KS)
    for r in range(KS - 1):
        ab = np.array([rr_pair(r, k, KS) for k in range(KS // 2)])
        a, b = ab[:, 0], ab[:, 1]
        apq = S[a, b]
        c, s = np.ones(KS // 2), np.zeros(KS // 2)
        rot = np.abs(apq) > tau
        d = S[b, b] - S[a, a]
        p2 = 2.0 * apq
        t = np.where(rot, p2 / np.where(rot, d + np.copysign(np.sqrt(d * d + p2 * p2), d), 1.0), 0.0)
        c = np.where(rot, 1.0 / np.sqrt(t * t + 1.0), 1.0)
        s = t * c
        G = np.eye(KS)
        G[a, a], G[a, b], G[b, a], G[b, b] = c, s, -s, c   # columns: [a, b] <- [c a - s b, s a + c b]
        S = G.T @ S @ G
        S = 0.5 * (S + S.T)
        Q = Q @ G
    return S, Q


def block_jacobi(A, max_sweeps=60):
    n = A.shape[0]
    assert n % KS == 0
    nb = n // KB
    A = A.copy()
    V = np.eye(n)
    tau = 1e-14 * np.linalg.norm(A)
    for sweep in range(1, max_sweeps + 1):
        rotated = False
        for r in range(nb - 1):
            J = np.eye(n)
            for k in range(nb // 2):
                I, Jb = rr_pair(r, k, nb)
                idx = np.r_[I * KB:(I + 1) * KB, Jb * KB:(Jb + 1) * KB]
                S = A[np.ix_(idx, idx)]
                off = S - np.diag(np.diag(S))
                if np.abs(off).max() <= tau:
                    continue
                rotated = True
                _, Q = inner_sweep(S, 0.25 * tau)
                J[np.ix_(idx, idx)] = Q
            A = J.T @ A @ J
            A = 0.5 * (A + A.T)
            V = V @ J
        if not rotated:
            return np.diag(A).copy(), V, sweep
    raise RuntimeError("no convergence")


def test_model_converges_to_lapack_eigenpairs():
    rng = np.random.default_rng(3)
    n = 128
    X = rng.standard_normal((n, 3 * n))
    A = -(X @ X.T) / (3 * n)          # chi0-like: negative semidefinite, clustered spectrum
    A[np.arange(n), np.arange(n)] += 0.05 * rng.standard_normal(n)
    lam, V, sweeps = block_jacobi(A)
    ref = np.linalg.eigvalsh(A)
    scale = np.abs(ref).max()
    assert np.abs(np.sort(lam) - ref).max() < 1e-13 * scale
    assert np.abs(V.T @ V - np.eye(n)).max() < 1e-13
    assert np.abs(A @ V - V * lam).max() < 1e-12 * scale
    assert sweeps <= 12


def test_zero_padding_gives_zero_eigenpairs():
    rng = np.random.default_rng(4)
    n, m = 128, 100                   # the device pads to a multiple of 64 with zeros
    X = rng.standard_normal((m, m))
    A = np.zeros((n, n))
    A[:m, :m] = X + X.T
    lam, V, _ = block_jacobi(A)
    ref = np.linalg.eigvalsh(A[:m, :m])
    small = np.abs(lam) <= 1e-12 * np.abs(ref).max()
    assert np.sum(small) == n - m                       # the padding contributes zero eigenvalues only
    assert np.abs(np.sort(lam[~small]) - ref).max() < 1e-13 * np.abs(ref).max()
    assert np.abs(V[m:, ~small]).max() < 1e-13         # and the kept eigenvectors vanish on it
