"""CPU: the learned-form checkers.  The FP64 MLP oracle's analytic gradient is
pinned by central finite differences; the dense Hamiltonian builder used to
check the device Lanczos is pinned by the state-vector oracle's Pauli
expectation; the sample layout (features / mask) is fixed."""
import numpy as np

import oracle
from logosq_b200 import abi, learned, workloads


def test_mlp_oracle_gradient_matches_finite_differences():
    shape = (7, 9, 2, 5)
    npar = oracle.mlp_num_params(*shape)
    assert npar == 7 * 9 + 9 + 9 * 9 + 9 + 9 * 5 + 5
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.4, npar)
    x = rng.normal(0, 1, (4, 7)).astype(np.float32)
    t = rng.uniform(-3, 3, (4, 5)).astype(np.float32)
    m = (rng.uniform(size=(4, 5)) < 0.7).astype(np.float32)
    loss, g = oracle.mlp_loss_grad(shape, p, x, t, m)
    assert loss > 0
    h = 1e-6
    fd = np.zeros(npar)
    for i in range(npar):
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd[i] = (oracle.mlp_loss_grad(shape, pp, x, t, m)[0] -
                 oracle.mlp_loss_grad(shape, pm, x, t, m)[0]) / (2 * h)
    assert np.abs(fd - g).max() < 1e-7 * max(1.0, np.abs(g).max())


def test_mlp_oracle_forward_consistent_with_loss():
    """The loss computed from mlp_forward's output equals the oracle's loss."""
    shape = (6, 8, 3, 4)
    rng = np.random.default_rng(1)
    p = rng.normal(0, 0.3, oracle.mlp_num_params(*shape)).astype(np.float32)
    x = rng.normal(0, 1, (3, 6)).astype(np.float32)
    t = rng.uniform(-1, 1, (3, 4)).astype(np.float32)
    m = np.ones((3, 4), dtype=np.float32)
    y = oracle.mlp_forward(shape, p, x)
    want = np.sum(1 - np.cos(y - t)) / m.sum()
    got, _ = oracle.mlp_loss_grad(shape, p.astype(np.float64), x, t, m)
    assert abs(got - want) < 1e-12


def test_dense_hamiltonian_matches_pauli_expectation():
    """For XX/YY/ZZ chains both Y conventions give the same operator; the dense
    matrix reproduces the oracle's Pauli expectation in both."""
    for n in (3, 5, 7):
        rec = workloads.heisenberg_instances(1, seed=n, n_lo=n, n_hi=n)[0]
        terms = learned.chain_terms(rec)
        H = oracle.dense_hamiltonian(n, terms)
        assert np.allclose(H, H.T)
        psi = workloads.gaussian_state(n, 3)
        got = float(np.real(np.vdot(psi, H @ psi)))
        assert abs(got - oracle.expectation(psi, terms, abi.Y_REFERENCE)) < 1e-12
        assert abs(got - oracle.expectation(psi, terms, abi.Y_TEXTBOOK)) < 1e-12


def test_sample_layout():
    rec = workloads.disordered_chains(1, seed=3, n_lo=12, n_hi=12)[0]
    f = learned.features(rec)
    assert f.shape == (46,) and f.dtype == np.float32
    assert np.allclose(f[0:33:3], rec["jx"]) and np.allclose(f[1:33:3], rec["jy"])
    assert np.allclose(f[2:33:3], rec["jz"]) and f[45] == np.float32(rec["h"])
    assert not f[33:45].any()
    m = learned.angle_mask(12)
    assert m.sum() == 96 and m[:96].all()
    s = learned.fixed_start(12)
    assert s.shape == (96,) and np.abs(s).max() <= 0.1
    assert np.array_equal(s, learned.fixed_start(12))


def test_disordered_chains_spread():
    recs = workloads.disordered_chains(50, seed=5, n_lo=12, n_hi=16, disorder=0.2)
    assert {r["n"] for r in recs} <= set(range(12, 17))
    for r in recs:
        for a in ("jx", "jy", "jz"):
            assert len(r[a]) == r["n"] - 1
            assert np.ptp(r[a]) <= 0.4 + 1e-12  # per-bond spread within +-disorder


def test_iterations_to():
    tr = np.array([[3.0, 2.0, 1.0005, 1.0], [5.0, 4.0, 3.0, 2.0]])
    it = learned.iterations_to(tr, np.array([1.0, 1.0]), 1e-3)
    assert list(it) == [2, 4]
