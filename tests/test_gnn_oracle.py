"""The CPU oracle of the initial-guess network: its analytic gradient agrees with
central finite differences (FP64, weights unrounded), and its graph has the
symmetric structure the CUDA backward pass relies on."""
import numpy as np

from adh_kraken_b200.mesh import small_delaunay_case
from oracle import gnn_oracle as go


def _setup(seed=0):
    case = small_delaunay_case(n=7, seed=3, nsteps=1)
    g = go.graph_arrays(case.xyz[:, :2], case.tri)
    rng = np.random.default_rng(seed)
    _, P = go.offsets()
    p = rng.normal(0, 0.2, P)
    F = rng.normal(0, 1, (case.nnodes, 8))
    T = rng.normal(0, 1, (case.nnodes, 3))
    return g, p, F, T


def test_graph_is_symmetric_with_reverse_slots():
    g, *_ = _setup()
    n = len(g["indptr"]) - 1
    row = np.repeat(np.arange(n), np.diff(g["indptr"]))
    assert np.array_equal(g["nbr"][g["rev"]], row)          # slot rev[s] of nbr[s] points back
    assert np.array_equal(row[g["rev"]], g["nbr"])
    assert np.all(np.diff(g["indptr"]) > 0)


def test_oracle_gradient_matches_finite_differences():
    g, p, F, T = _setup()
    loss, grad, _ = go.loss_and_grad(p, g, F, T, bf16=False)
    rng = np.random.default_rng(1)
    idx = rng.choice(len(p), 60, replace=False)
    eps = 1e-6
    for k in idx:
        pp, pm = p.copy(), p.copy()
        pp[k] += eps; pm[k] -= eps
        fd = (go.loss_and_grad(pp, g, F, T, bf16=False)[0] - go.loss_and_grad(pm, g, F, T, bf16=False)[0]) / (2 * eps)
        assert abs(fd - grad[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, grad[k])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.14159], np.float32)
    r = go.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0                       # tie -> even
    assert r[2] == np.float32(1.0 + 2 ** -7)                 # above the tie -> up
    assert r[3] == -2.5
    assert abs(r[4] - 3.140625) < 1e-7
