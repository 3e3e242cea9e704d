"""The dense adjoint reference (oracle/adjoint_dense.py) checked on the CPU: the SO(3) left
Jacobian it uses is the derivative of the exponential, its gradient is the gradient of the robust
cost in the solver's local coordinates, and its Hessian is symmetric."""
import numpy as np
import pytest

from oracle.adjoint_dense import Problem, so3_exp, so3_left_jacobian
from typecv_b200 import synthetic as S


def small_problem(seed=4, cameras=4, points=40):
    sc = S.helix_scene(seed=seed, cameras=cameras, points=points, laps=0.25)
    s, i = sc.packed()
    return Problem(sc.C, sc.P, sc.M, s, i)


def test_left_jacobian_is_the_derivative_of_the_exponential():
    rng = np.random.default_rng(0)
    w = rng.normal(size=3) * 0.3
    a = rng.normal(size=3)
    h = 1e-6
    num = np.zeros((3, 3))
    for j in range(3):
        e = np.zeros(3)
        e[j] = h
        num[:, j] = (so3_exp(w + e) @ a - so3_exp(w - e) @ a) / (2 * h)
    A = so3_exp(w) @ a
    K = np.array([[0, -A[2], A[1]], [A[2], 0, -A[0]], [-A[1], A[0], 0]])
    assert np.allclose(num, -K @ so3_left_jacobian(w), atol=1e-8)


def test_gradient_matches_central_differences_of_the_cost():
    pb = small_problem()
    rng = np.random.default_rng(1)
    delta = rng.normal(size=pb.n) * 1e-3
    g = pb.gradient(delta)
    h = 1e-6
    for j in rng.choice(pb.n, 12, replace=False):
        e = np.zeros(pb.n)
        e[j] = h
        num = (pb.half_cost(delta + e) - pb.half_cost(delta - e)) / (2 * h)
        assert abs(num - g[j]) <= 1e-5 * max(1.0, abs(g[j]))


def test_hessian_is_symmetric():
    pb = small_problem(cameras=3, points=12)
    H = np.zeros((pb.n, pb.n))
    e = np.zeros(pb.n)
    for j in range(pb.n):
        e[j] = 1e-6
        H[:, j] = (pb.gradient(e) - pb.gradient(-e)) / 2e-6
        e[j] = 0
    assert np.max(np.abs(H - H.T)) <= 1e-5 * np.max(np.abs(H))
