"""The seeded problem generators (CPU)."""
import numpy as np
import pytest

import problems as P


def test_heat3d_32_matches_reference_sizes():
    """7-point 32^3 Laplacian: n = 32768, nnz = 223232, upper nnz = 128000."""
    s = P.heat3d(32, sigma=0.0, seed=0)
    assert (s.n, s.nnz, s.upper().nnz) == (32768, 223232, 128000)
    A = s.to_scipy()
    assert abs(A - A.T).max() == 0
    assert np.allclose(A.diagonal(), 6.0)
    # diagonal first in every row, others ascending
    assert all(s.ja[s.ia[i]] == i for i in range(0, s.n, 997))
    assert np.all(s.rhs >= -1) and np.all(s.rhs < 1)


def test_heat3d_size_formula_for_128():
    n = 128 ** 3
    assert 7 * n - 6 * 128 ** 2 == 14581760


def test_heat3d_lognormal_is_deterministic_and_spd():
    a = P.heat3d(10, 9, 8, sigma=1.5, seed=4)
    b = P.heat3d(10, 9, 8, sigma=1.5, seed=4)
    assert np.array_equal(a.a, b.a) and np.array_equal(a.rhs, b.rhs)
    A = a.to_scipy()
    assert abs(A - A.T).max() < 1e-12
    d = np.asarray(A.diagonal())
    off = np.asarray(abs(A).sum(axis=1)).ravel() - d
    assert np.all(d >= off - 1e-12)  # diagonally dominant


def test_heat2d_batch_is_block_diagonal():
    s = P.heat2d_batch(12, 8, 24, 1.0, 3)
    assert len(s.parts) == 13 and s.parts[-1] == s.n
    sides = np.sqrt(np.diff(s.parts)).round().astype(int)
    assert np.all(sides >= 8) and np.all(sides <= 24)
    rows = np.repeat(np.arange(s.n), np.diff(s.ia))
    part = np.searchsorted(s.parts, rows, side="right") - 1
    part_c = np.searchsorted(s.parts, s.ja, side="right") - 1
    assert np.array_equal(part, part_c)


def test_lame3d_clamped_symmetric():
    s = P.lame3d(6, 0.3, 1.0, 1)
    assert s.bs == 3 and s.n == 216
    A = s.to_scipy()
    assert abs(A - A.T).max() < 1e-12 * abs(A).max()
    # clamped z = 0 layer: identity rows, zero load
    for node in range(36):
        r = A[3 * node:3 * node + 3].toarray()
        assert np.allclose(r[:, 3 * node:3 * node + 3], np.eye(3))
        assert np.count_nonzero(r) == 3
    assert np.allclose(s.rhs[0][:108], 0.0)
    assert s.rhs[0][2::3][36:].max() < 0  # body load points down
    # positive definite on the free nodes
    free = A[108:, 108:].toarray()
    assert np.linalg.eigvalsh(free).min() > 0


def test_lame_periodic_six_load_cases():
    s = P.lame_periodic(10, 0.3, 1.5, 2.5, 0.2, 100.0, 2)
    assert s.rhs.shape == (6, 3 * s.n)
    assert s.info["frac"] >= 0.2 or s.info["count"] > 0
    A = s.to_scipy()
    assert abs(A - A.T).max() < 1e-10 * abs(A).max()
    assert np.linalg.eigvalsh(A.toarray()).min() > 0  # node 0 pinned: no rigid modes
    # every node row has 27 blocks (periodic stencil) except the pinned node
    counts = np.diff(s.ia)
    assert counts[0] == 1 and np.all(counts[1:] <= 27)


@pytest.mark.parametrize("k", [1])
def test_config_one(k):
    s = P.config(k)
    assert s.n == 32768
