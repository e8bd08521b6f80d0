"""CPU: the FP64 reference of the scheduler network (oracle/mlp_oracle.py) against
central finite differences, so the GPU gradient check compares with a verified oracle."""
import numpy as np

from oracle import mlp_oracle as M
from starplat_b200 import _lib


def test_parameter_count_matches_the_library():
    assert M.H * M.IN + M.H * M.H + 3 * M.H + 1 == _lib.SP_MLP_PARAMS


def test_oracle_gradient_finite_differences():
    rng = np.random.default_rng(0)
    P = _lib.SP_MLP_PARAMS
    p = rng.normal(0, 0.3, P)
    X = rng.normal(0, 1, (40, M.IN))
    T = rng.normal(0, 1, 40)
    L, g = M.loss_grad(p, X, T)
    idx = rng.choice(P, 60, replace=False)
    eps = 1e-6
    for i in idx:
        d = np.zeros(P)
        d[i] = eps
        num = (M.loss_grad(p + d, X, T)[0] - M.loss_grad(p - d, X, T)[0]) / (2 * eps)
        assert abs(num - g[i]) <= 1e-6 * max(1.0, abs(num)), (i, num, g[i])
