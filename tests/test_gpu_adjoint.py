"""The eigenvector adjoint on the GPU (sa_adjoint) against the dense FP64 oracle and finite
differences: the smoothed-energy gradient per vertex and in alpha, the eigenvector tangent, the
torch.autograd.Function, and the tangent predictor in a sweep."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import adjoint_oracle as AO  # noqa: E402
from oracle import specann_oracle as O  # noqa: E402
from specann_b200 import graphs  # noqa: E402
from specann_b200.differentiation import EigenProblem, smoothed_energy  # noqa: E402
from specann_b200.spectral_annealing import SpectralAnnealing  # noqa: E402


@pytest.fixture(scope="module")
def J12():
    # BA(n = 2^12, m = 20) with +-1 couplings, the dense-check size of the differentiation workload
    return graphs.barabasi_albert(1 << 12, 20, seed=4096, couplings="pm1")


@pytest.fixture(scope="module")
def dense12(J12):
    return {alpha: AO.energy_gradient(J12, alpha, 8.0) for alpha in (0.3, 0.7)}


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


# (precision, Lanczos tolerance, MINRES tolerance, bound on the relative gradient error): the
# adjoint is resolved to about the eigenpair's own accuracy, not below it
@pytest.mark.parametrize("precision,tol,adj_tol,bound", [(64, 1e-10, 1e-8, 1e-6), (32, 1e-6, 1e-4, 2e-3)])
@pytest.mark.parametrize("alpha", [0.3, 0.7])
def test_gradient_matches_dense_oracle(J12, dense12, precision, tol, adj_tol, bound, alpha):
    L_ref, g_ref, lam_ref, _ = dense12[alpha]
    prob = EigenProblem(J12, precision=precision)
    L, grad, dalpha, res = prob.energy_and_gradient(alpha, beta=8.0, tol=tol, adj_tol=adj_tol)
    print(f"precision {precision} alpha {alpha}: minres {res.iterations} it, residual {res.residual:.2e}, "
          f"grad rel err {rel(grad.cpu().numpy(), g_ref):.2e}")
    assert res.status == 0, (res.status, res.iterations, res.residual)
    assert L == pytest.approx(L_ref, rel=bound)
    g = grad.cpu().numpy()
    assert rel(g, g_ref) < bound
    assert dalpha == pytest.approx(g_ref.sum(), rel=bound)
    prob.close()


def test_tangent_matches_dense_oracle(J12):
    alpha = 0.55
    t_ref, lam_ref, y_ref = AO.eigvec_tangent(J12, alpha)
    prob = EigenProblem(J12, precision=64)
    lam, y = prob.eigenpair(alpha, tol=1e-10)
    assert lam == pytest.approx(lam_ref, abs=1e-10)
    t, res = prob.tangent(alpha, lam, y, tol=1e-8)
    assert res.status == 0, (res.status, res.iterations, res.residual)
    sgn = np.sign(float(y.cpu().numpy() @ y_ref))
    assert rel(sgn * t.cpu().numpy(), t_ref) < 1e-5
    prob.close()


def test_autograd_function_and_offsets(J12, dense12):
    prob = EigenProblem(J12, precision=64)
    alpha = torch.tensor(0.3, dtype=torch.float64, requires_grad=True)
    offsets = torch.zeros(J12.shape[0], dtype=torch.float64, device="cuda", requires_grad=True)
    L = smoothed_energy(prob, alpha, offsets, beta=8.0, tol=1e-10, adj_tol=1e-8)
    L.backward()
    _, g_ref, _, _ = dense12[0.3]
    assert float(alpha.grad) == pytest.approx(g_ref.sum(), rel=1e-6)
    assert rel(offsets.grad.cpu().numpy(), g_ref) < 1e-6
    # per-vertex offsets move the operator: L(a + h v) - L(a - h v) / 2h = grad . v
    v = torch.tensor(np.random.default_rng(3).standard_normal(J12.shape[0]), device="cuda")
    h = 1e-5
    Lp = smoothed_energy(prob, torch.tensor(0.3, dtype=torch.float64), h * v, tol=1e-10, adj_tol=1e-2)
    Lm = smoothed_energy(prob, torch.tensor(0.3, dtype=torch.float64), -h * v, tol=1e-10, adj_tol=1e-2)
    fd = float(Lp - Lm) / (2 * h)
    assert float(offsets.grad @ v) == pytest.approx(fd, rel=1e-3)
    prob.close()


def test_gradient_in_alpha_matches_fd_at_2e18():
    # the differentiation workload: BA(2^18, m = 20), +-1 couplings, beta = 8, central FD h = 1e-4
    J = graphs.barabasi_albert(1 << 18, 20, seed=42, couplings="pm1")
    prob = EigenProblem(J, precision=64)
    alpha, h = 0.5, 1e-4
    _, _, dalpha, res = prob.energy_and_gradient(alpha, beta=8.0, tol=1e-10, adj_tol=1e-8)
    assert res.status == 0, (res.status, res.iterations, res.residual)
    Lp, _, _, _ = prob.energy_and_gradient(alpha + h, beta=8.0, tol=1e-10, adj_tol=1e-3)
    Lm, _, _, _ = prob.energy_and_gradient(alpha - h, beta=8.0, tol=1e-10, adj_tol=1e-3)
    fd = (Lp - Lm) / (2 * h)
    print(f"2^18: dL/dalpha adjoint {dalpha:.8e} FD {fd:.8e} minres {res.iterations} it")
    assert dalpha == pytest.approx(fd, rel=1e-2)
    prob.close()


def test_tangent_predictor_sweep():
    J = graphs.barabasi_albert(1 << 13, 10, seed=5, couplings="pm1")
    s = SpectralAnnealing("t.txt", "t", random_seed=42, num_alphas=24, pred_mode="tangent", write_results=False)
    e, spins, _ = s.solve(J)
    assert O.exact_energy(J, spins) == e
    rows = s.alpha_results
    assert all(r["eigsh_converged"] for r in rows)
    assert sum(1 for r in rows if r["pred_accepted"]) >= len(rows) // 2
    assert all(r["tangent_spmvs"] > 0 for r in rows)
