"""The collision the kernels use against the reference's MRT operators.

The kernels (lbflow_b200/csrc/kernels.cuh, collide_trt) apply the reference's
MRT (scsp.cpp:411-464, colorfluid.cpp:360-387) as a two-rate update of
opposite-direction pairs.  These checks take M, M^-1 and S from the C oracle
(whose tables reproduce the reference bit for bit) and confirm, for random
states, forces and relaxation times, that
M^-1 S M (feq - f) + M^-1 (I - S/2) M S_guo equals the two-rate form to
round-off, and that the moment identities of scripts/moment_audit.py:19-73 hold.
"""
import numpy as np
import pytest

from oracle_port import mrt_tables

E19 = np.array([(0, 0, 0), (0, 0, 1), (0, 0, -1), (0, 1, 0), (0, -1, 0), (1, 0, 0), (-1, 0, 0),
                (0, 1, 1), (0, 1, -1), (0, -1, 1), (0, -1, -1), (1, 0, 1), (1, 0, -1), (-1, 0, 1),
                (-1, 0, -1), (1, 1, 0), (1, -1, 0), (-1, 1, 0), (-1, -1, 0)], float)
W19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
E9 = np.array([(0, 0), (0, 1), (1, 0), (0, -1), (-1, 0), (1, 1), (1, -1), (-1, -1), (-1, 1)], float)
W9 = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)


def lattice(q):
    E, W = (E19, W19) if q == 19 else (E9, W9)
    op = [int(np.where((E == -E[k]).all(1))[0][0]) for k in range(q)]
    return E, W, op


def two_rate(f, feq, src, op, sp, sm):
    fp, fm = (f + f[op]) / 2, (f - f[op]) / 2
    ep, em = (feq + feq[op]) / 2, (feq - feq[op]) / 2
    gp, gm = (src + src[op]) / 2, (src - src[op]) / 2
    return f - sp * (fp - ep) - sm * (fm - em) + (1 - sp / 2) * gp + (1 - sm / 2) * gm


@pytest.mark.parametrize('q', [9, 19])
@pytest.mark.parametrize('tau', [0.51, 0.6, 0.8, 1.0, 1.4, 3.0])
def test_mrt_equals_two_rate_form(q, tau):
    E, W, op = lattice(q)
    M, Mi, S = mrt_tables(q, tau)
    su = 1 / tau
    sm = 8 * (2 - su) / (8 - su)
    rng = np.random.default_rng(q * 100 + int(tau * 10))
    for _ in range(50):
        rho0 = 1.0
        f = W * (1 + 1e-2 * rng.standard_normal(q))
        F = 1e-4 * rng.standard_normal(E.shape[1])
        rho, u = f.sum(), E.T @ f / rho0 + F / (2 * rho0)
        eu = E @ u
        feq = W * (rho + rho0 * (3 * eu + 4.5 * eu ** 2 - 1.5 * u @ u))
        ef = E @ F
        src = W * (3 * (ef - u @ F) + 9 * eu * ef)
        ref = f + Mi @ (S * (M @ (feq - f))) + Mi @ ((1 - 0.5 * S) * (M @ src))
        got = two_rate(f, feq, src, op, su, sm)
        assert np.max(np.abs(got - ref) / np.abs(ref)) < 1e-14


@pytest.mark.parametrize('q', [9, 19])
def test_moment_identities(q):
    """scripts/moment_audit.py:35-55 on the oracle's (= the reference's) tables."""
    E, W, op = lattice(q)
    M, Mi, S = mrt_tables(q, 1.2)
    assert np.max(np.abs(M @ Mi - np.eye(q))) < 3e-14
    assert abs(W.sum() - 1) < 3e-14
    assert np.max(np.abs(W @ E)) < 3e-14
    assert np.max(np.abs(np.einsum('q,qa,qb->ab', W, E, E) - np.eye(E.shape[1]) / 3)) < 3e-14
    # Rate classes: conserved rows are mass and momentum; the rest split by parity.
    even = np.array([np.array_equal(M[k], M[k][op]) for k in range(q)])
    cons = S == 0
    assert cons.sum() == 1 + E.shape[1]
    su, sq = 1 / 1.2, 8 * (2 - 1 / 1.2) / (8 - 1 / 1.2)
    assert np.allclose(S[even & ~cons], su) and np.allclose(S[~even & ~cons], sq)
