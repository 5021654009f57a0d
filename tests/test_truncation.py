"""Block-matrix truncation (svd_truncate / heev_truncate, block_matrix_algorithms.h:136-355):
the oracle pinned against a numpy restatement on the CPU, the device C-ABI against the oracle."""
import numpy as np
import pytest

from oracle.oracle import truncate_heev as orc_heev
from oracle.oracle import truncate_svd as orc_svd


def estimate_truncation(vals, Mmax, cutoff):
    """block_matrix_algorithms.h:136-183: keep values >= max(cutoff * s_max, s_sorted[Mmax])."""
    allv = np.sort(np.concatenate(vals))[::-1]
    cut = cutoff * allv[0]
    if allv.size > Mmax:
        cut = max(cut, allv[Mmax])
    dropped = allv[allv < cut]
    res = {"smallest_ev": cut / allv[0], "truncated_fraction": dropped.sum() / allv.sum(),
           "truncated_weight": (dropped ** 2).sum() / (allv ** 2).sum()}
    keep = [int(np.argmax(v < cut)) if (v < cut).any() else v.size for v in vals]
    res["bond_dimension"] = sum(keep)
    return keep, res


def random_blocks(rng, shapes, rank=None):
    out = []
    for i, (m, n) in enumerate(shapes):
        if rank and rank[i] is not None:
            out.append(rng.standard_normal((m, rank[i])) @ rng.standard_normal((rank[i], n)))
        else:
            out.append(rng.standard_normal((m, n)))
    return out


CASES = {
    # shapes, rank per block (None = full), Mmax, cutoff
    "mixed": ([(40, 30), (17, 52), (64, 64), (1, 9), (12, 1), (5, 5)], None, 60, 1e-16),
    # zero singular values come out at ~1e-15 s_max: the cutoff drops them (at 1e-16 whether a
    # rounding-level value survives would depend on the SVD algorithm)
    "rank_deficient": ([(30, 20), (25, 40), (10, 10)], [4, None, 0], 200, 1e-12),
    "cutoff": ([(50, 40), (20, 20)], None, 1000, 1e-1),
    # work matrices larger than the shared-memory path
    "global_path": ([(200, 180), (33, 300), (7, 7)], None, 150, 1e-16),
    # a block whose work matrix fits in shared memory but not together with its rotations (hybrid
    # placement), in one launch with blocks that fit entirely
    "hybrid_path": ([(174, 109), (120, 110), (5, 5)], None, 250, 1e-16),
}


def check_svd(out, res, blocks, keep_ref, S_ref, res_ref, tol):
    assert [o[1].size for o in out] == keep_ref
    assert res["bond_dimension"] == res_ref["bond_dimension"]
    for f in ("truncated_weight", "truncated_fraction", "smallest_ev"):
        assert abs(res[f] - res_ref[f]) <= 1e-12 * max(1.0, abs(res_ref[f])) + 1e-15, f
    smax = max(np.linalg.svd(b, compute_uv=False)[0] for b in blocks if b.size)
    for (U, S, Vt), s_ref, b in zip(out, S_ref, blocks):
        k = S.size
        assert np.allclose(S, s_ref[:k], rtol=0, atol=tol * smax)
        if k:
            assert np.abs(U.T @ U - np.eye(k)).max() < tol * 10
            assert np.abs(Vt @ Vt.T - np.eye(k)).max() < tol * 10
            # the kept part of the block: U S Vt is the best rank-k approximation
            full_u, full_s, full_vt = np.linalg.svd(b, full_matrices=False)
            best = (full_u[:, :k] * full_s[:k]) @ full_vt[:k]
            assert np.abs((U * S) @ Vt - best).max() < tol * 100 * smax


@pytest.mark.parametrize("case", list(CASES))
def test_oracle_svd_truncate_matches_numpy(case):
    shapes, rank, Mmax, cutoff = CASES[case]
    rng = np.random.default_rng(7)
    blocks = random_blocks(rng, shapes, rank)
    out, res = orc_svd(blocks, Mmax, cutoff)
    S_ref = [np.linalg.svd(b, compute_uv=False) for b in blocks]
    keep_ref, res_ref = estimate_truncation(S_ref, Mmax, cutoff)
    check_svd(out, res, blocks, keep_ref, S_ref, res_ref, 1e-12)


def test_oracle_heev_truncate_matches_numpy():
    rng = np.random.default_rng(3)
    blocks = []
    for n, r in ((30, 30), (12, 5), (40, 40), (3, 3)):
        a = rng.standard_normal((n, r))
        blocks.append(a @ a.T)
    Mmax, cutoff = 50, 1e-14
    out, res = orc_heev(blocks, Mmax, cutoff)
    w_ref = [np.linalg.eigvalsh(b)[::-1] for b in blocks]
    keep_ref, res_ref = estimate_truncation([np.where(w > 0, np.sqrt(np.abs(w)), w) for w in w_ref], Mmax, cutoff)
    assert [o[1].size for o in out] == keep_ref
    assert res["bond_dimension"] == res_ref["bond_dimension"]
    # heev_truncate takes sqrt of the positive eigenvalues: rounding-level eigenvalues of the
    # rank-deficient block (~1e-16 |w0|) enter the sums as ~1e-8 |w0|^(1/2), so the fractions
    # agree to ~1e-8 relative, not to rounding
    assert abs(res["truncated_weight"] - res_ref["truncated_fraction"]) < 1e-6 * res_ref["truncated_fraction"]
    assert res["truncated_weight"] == res["truncated_fraction"]  # fraction in both fields
    for (U, ev), w, b in zip(out, w_ref, blocks):
        assert np.allclose(ev, w[:ev.size], atol=1e-10 * abs(w[0]))
        if ev.size:
            assert np.abs(b @ U - U * ev).max() < 1e-9 * abs(w[0])


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(CASES))
def test_device_svd_truncate_matches_oracle(gpu_ctx, case):
    from qcmaquis_b200.dmrg import truncate_svd
    shapes, rank, Mmax, cutoff = CASES[case]
    rng = np.random.default_rng(11)
    blocks = random_blocks(rng, shapes, rank)
    ref, res_ref = orc_svd(blocks, Mmax, cutoff)
    out, res = truncate_svd(gpu_ctx, blocks, Mmax, cutoff)
    check_svd(out, res, blocks, [o[1].size for o in ref], [o[1] for o in ref], res_ref, 1e-12)
    # singular vectors agree with LAPACK's column by column up to sign (the spectra have no ties)
    for (U, S, Vt), (Ur, Sr, Vtr) in zip(out, ref):
        for j in range(S.size):
            sg = np.sign(U[:, j] @ Ur[:, j])
            assert np.abs(U[:, j] - sg * Ur[:, j]).max() < 1e-8
            assert np.abs(Vt[j] - sg * Vtr[j]).max() < 1e-8


def middle_bond_blocks(seed=1):
    """44 blocks shaped like the two-site tensor's at the L=24, M=512 middle bond (up to 178 x 114), each with
    its own exponentially decaying spectrum and scale (no ties across blocks)."""
    rng = np.random.default_rng(seed)
    shapes = [(178, 114), (160, 120), (150, 100), (114, 140)] + [(int(rng.integers(20, 140)), int(rng.integers(16, 110)))
                                                                 for _ in range(40)]
    blocks = []
    for (m, n) in shapes:
        k = min(m, n)
        U, _ = np.linalg.qr(rng.standard_normal((m, k)))
        V, _ = np.linalg.qr(rng.standard_normal((n, k)))
        s = rng.uniform(0.5, 2.0) * np.exp(-np.arange(k) * rng.uniform(0.15, 0.4))
        blocks.append((U * s) @ V.T)
    return blocks


@pytest.mark.gpu
def test_device_svd_truncate_middle_bond_blocks(gpu_ctx):
    """The truncation SVD (pivoted QR, Jacobi on R^T) on blocks of the bench bond's sizes and graded spectra,
    against the oracle (LAPACK): kept dimensions, singular values, kept singular vectors up to sign."""
    from qcmaquis_b200.dmrg import truncate_svd
    blocks = middle_bond_blocks()
    ref, res_ref = orc_svd(blocks, 512, 1e-16)
    out, res = truncate_svd(gpu_ctx, blocks, 512, 1e-16)
    check_svd(out, res, blocks, [o[1].size for o in ref], [o[1] for o in ref], res_ref, 1e-12)
    for (U, S, Vt), (Ur, Sr, Vtr) in zip(out, ref):
        for j in range(S.size):
            sg = np.sign(U[:, j] @ Ur[:, j])
            assert np.abs(U[:, j] - sg * Ur[:, j]).max() < 1e-8
            assert np.abs(Vt[j] - sg * Vtr[j]).max() < 1e-8


@pytest.mark.gpu
def test_device_svd_truncate_degenerate(gpu_ctx):
    """Orthogonal blocks (all singular values 1) and a scaled copy: the cut falls in the gap."""
    from qcmaquis_b200.dmrg import truncate_svd
    rng = np.random.default_rng(5)
    q1, _ = np.linalg.qr(rng.standard_normal((24, 24)))
    q2, _ = np.linalg.qr(rng.standard_normal((30, 16)))
    blocks = [q1, 0.5 * q2, 1e-3 * rng.standard_normal((8, 9))]
    # Mmax = 39: the cut s[39] is the smallest of the sixteen 0.5s, so the tied cluster is kept whole
    out, res = truncate_svd(gpu_ctx, blocks, 39, 1e-16)
    assert [o[1].size for o in out] == [24, 16, 0]
    assert res["bond_dimension"] == 40
    for (U, S, Vt), b in zip(out[:2], blocks[:2]):
        assert np.abs((U * S) @ Vt - b).max() < 1e-13
    # Mmax = 40: values >= s[40] are kept, s[40] itself included (estimate_truncation keeps Mmax + 1)
    out, res = truncate_svd(gpu_ctx, blocks, 40, 1e-16)
    assert [o[1].size for o in out] == [24, 16, 1]


@pytest.mark.gpu
def test_device_heev_truncate_matches_oracle(gpu_ctx):
    from qcmaquis_b200.dmrg import truncate_heev
    rng = np.random.default_rng(9)
    blocks = []
    for n, r in ((30, 30), (12, 5), (64, 64), (3, 3), (1, 1)):
        a = rng.standard_normal((n, r))
        blocks.append(a @ a.T)
    Mmax, cutoff = 70, 1e-14
    ref, res_ref = orc_heev(blocks, Mmax, cutoff)
    out, res = truncate_heev(gpu_ctx, blocks, Mmax, cutoff)
    assert [o[1].size for o in out] == [o[1].size for o in ref]
    assert res["bond_dimension"] == res_ref["bond_dimension"]
    # fractions: sqrt of rounding-level eigenvalues of the rank-deficient block (see above)
    for f in ("truncated_weight", "truncated_fraction"):
        assert abs(res[f] - res_ref[f]) <= 1e-6 * abs(res_ref[f]) + 1e-12, f
    assert abs(res["smallest_ev"] - res_ref["smallest_ev"]) <= 1e-12
    for (U, ev), (Ur, evr), b in zip(out, ref, blocks):
        assert np.allclose(ev, evr, rtol=0, atol=1e-11 * abs(evr[0]) if evr.size else 0)
        if ev.size:
            assert np.abs(b @ U - U * ev).max() < 1e-9 * abs(ev[0])
            assert np.abs(np.abs(np.diag(U.T @ Ur)) - 1).max() < 1e-8


@pytest.mark.gpu
@pytest.mark.parametrize("lq", [False, True])
def test_qr_blocks_householder(gpu_ctx, lq):
    """Batched thin QR / LQ (one launch for all blocks): tall, wide, square, 1 x n, n x 1, rank-deficient and
    zero blocks; A = QR (LQ), orthonormal Q, triangular R (L), and R's diagonal equal to LAPACK's (numpy's
    Householder QR: the same reflector convention beta = -sign(alpha) |x|) up to rounding."""
    from qcmaquis_b200.dmrg import qr_blocks
    rng = np.random.default_rng(3)
    shapes = [(40, 12), (12, 40), (33, 33), (1, 7), (7, 1), (300, 90), (64, 200)]
    blocks = [rng.standard_normal(s) for s in shapes]
    blocks.append(np.outer(rng.standard_normal(20), rng.standard_normal(9)))  # rank 1
    blocks.append(np.ones((6, 4)))                                             # the const state's blocks
    out = qr_blocks(gpu_ctx, blocks, lq=lq)
    for A, (X, Y) in zip(blocks, out):
        m, n = A.shape
        k = min(m, n)
        if lq:
            L, Q = X, Y
            assert L.shape == (m, k) and Q.shape == (k, n)
            assert np.abs(L @ Q - A).max() <= 1e-13 * max(1.0, np.abs(A).max())
            assert np.abs(Q @ Q.T - np.eye(k)).max() < 1e-13
            assert np.abs(np.triu(L[:k, :k], 1)).max() == 0.0
            ref = np.linalg.qr(A.T, mode="r")
            assert np.allclose(np.diag(L[:k, :k]), np.diag(ref[:k, :k]), rtol=1e-10, atol=1e-12)
        else:
            Q, R = X, Y
            assert Q.shape == (m, k) and R.shape == (k, n)
            assert np.abs(Q @ R - A).max() <= 1e-13 * max(1.0, np.abs(A).max())
            assert np.abs(Q.T @ Q - np.eye(k)).max() < 1e-13
            assert np.abs(np.tril(R[:, :k], -1)).max() == 0.0
            ref = np.linalg.qr(A, mode="r")
            assert np.allclose(np.diag(R[:, :k]), np.diag(ref[:k, :k]), rtol=1e-10, atol=1e-12)
