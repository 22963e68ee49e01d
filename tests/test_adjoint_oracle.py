"""The dense differentiation oracle (oracle/adjoint_oracle.py) against finite differences: the
adjoint formula for dL/dalpha and dL/da (directional), and the eigenvector tangent dy/dalpha.
This pins the checker the GPU adjoint tests use. CPU only."""
import numpy as np
import pytest

from oracle import adjoint_oracle as AO
from specann_b200 import build, graphs


@pytest.fixture(scope="module")
def J():
    build.build_all()
    return graphs.barabasi_albert(300, 5, seed=11, couplings="pm1")


@pytest.mark.parametrize("alpha", [0.0, 0.35, 0.8])
@pytest.mark.parametrize("beta", [1.0, 8.0])
def test_gradient_sum_matches_fd_in_alpha(J, alpha, beta):
    L, grad, _, _ = AO.energy_gradient(J, alpha, beta)
    fd = AO.fd_alpha(J, alpha, beta, h=1e-5)
    assert grad.sum() == pytest.approx(fd, rel=1e-5, abs=1e-9 * max(1.0, abs(L)))


def test_per_vertex_gradient_matches_directional_fd(J):
    rng = np.random.default_rng(0)
    alpha, beta = 0.5, 8.0
    _, grad, _, _ = AO.energy_gradient(J, alpha, beta)
    for _ in range(3):
        v = rng.standard_normal(J.shape[0])
        fd = AO.fd_direction(J, alpha, v, beta, h=1e-6)
        assert grad @ v == pytest.approx(fd, rel=1e-5, abs=1e-9)


def test_tangent_matches_fd_of_eigenvector(J):
    alpha, h = 0.45, 1e-6
    t, lam, y = AO.eigvec_tangent(J, alpha)
    _, Mp, _, _ = AO._parts(J, alpha + h)
    _, Mm, _, _ = AO._parts(J, alpha - h)
    _, yp = AO.leading_pair(Mp)
    _, ym = AO.leading_pair(Mm)
    yp *= np.sign(yp @ y)
    ym *= np.sign(ym @ y)
    fd = (yp - ym) / (2 * h)
    assert abs(t @ y) < 1e-10
    assert np.linalg.norm(t - fd) <= 1e-5 * np.linalg.norm(fd)
