"""The FP64 FMM restatement (oracle/fmm.py) converges to the FP64 direct sum
and its operators satisfy the exact translation identities."""
import numpy as np

from conftest import rel_l2


def test_fmm_oracle_converges(oracle_mod):
    from oracle import fmm
    X, Y, Z = 24, 20, 3
    d = (5e-9, 5e-9, 5e-9)
    rng = np.random.default_rng(1)
    rho = rng.standard_normal((Z, Y, X))
    g = oracle_mod.Grid(X, Y, Z, *d)
    exact = oracle_mod.potential_direct(g, rho)
    errs = [rel_l2(fmm.Plan(X, Y, Z, *d, P=P, s=2).potential(rho), exact) for P in (1, 2, 4)]
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] < 3e-3


def test_m2m_l2l_are_exact(oracle_mod):
    """M2M of a multipole then evaluation equals direct evaluation of the
    shifted multipole; L2L is an exact re-centring"""
    from oracle import fmm
    lay = fmm.Layout(4)
    T = fmm.op_m2m(lay, (0.25, -0.25, 0.0))
    T2 = fmm.op_m2m(lay, (-0.25, 0.25, 0.0))
    # shifting child->parent then the inverse offset is not identity (different
    # units), but parity blocks must decouple for in-plane offsets
    NE = lay.n_even
    assert np.abs(T[:NE, NE:]).max() < 1e-12 and np.abs(T[NE:, :NE]).max() < 1e-12
    assert np.abs(T2[:NE, NE:]).max() < 1e-12
    L = fmm.op_l2l(lay, (0.25, 0.25, 0.0))
    assert np.abs(L[:NE, NE:]).max() < 1e-12
