"""GPU: learned warm start.  Device FP32 network vs the FP64 CPU oracle
(forward to 1e-5 relative, gradients to 1e-4 relative of the largest entry --
FP32 accumulation over K <= 256 terms), Adam against a numpy restatement,
FP64 Lanczos against numpy eigvalsh (1e-10), and the gain of a trained network
over random-init VQE on fresh chains."""
import numpy as np
import pytest

import oracle
from logosq_b200 import LogosQError, abi, learned, workloads

pytestmark = pytest.mark.gpu


def _data(rng, shape, batch):
    x = rng.normal(0, 1, (batch, shape[0])).astype(np.float32)
    t = rng.uniform(-3, 3, (batch, shape[3])).astype(np.float32)
    m = (rng.uniform(size=(batch, shape[3])) < 0.8).astype(np.float32)
    return x, t, m


@pytest.mark.parametrize("shape,batch", [((7, 9, 2, 5), 3), ((46, 256, 3, 128), 70),
                                         ((46, 256, 3, 128), 257)])
def test_mlp_forward_and_gradient_match_oracle(shape, batch):
    net = learned.WarmStartMLP(*shape, seed=3)
    assert net.num_params == oracle.mlp_num_params(*shape)
    rng = np.random.default_rng(batch)
    x, t, m = _data(rng, shape, batch)
    p = net.params()
    want = oracle.mlp_forward(shape, p, x)
    got = net.forward(x)
    assert np.abs(got - want).max() <= 1e-5 * max(1.0, np.abs(want).max())
    loss = net.loss_grad(x, t, m)
    want_loss, want_g = oracle.mlp_loss_grad(shape, p.astype(np.float64), x, t, m)
    assert abs(loss - want_loss) <= 1e-5 * want_loss
    g = net.grads()
    assert np.abs(g - want_g).max() <= 1e-4 * np.abs(want_g).max()
    net.close()


def test_mlp_backward_matches_loss_gradient():
    """lq_mlp_backward with dy = mask sin(y - t) / sum(mask) reproduces the angle
    loss gradient (same kernels, caller-supplied dL/dy)."""
    shape = (46, 256, 3, 128)
    net = learned.WarmStartMLP(*shape, seed=8)
    rng = np.random.default_rng(2)
    x, t, m = _data(rng, shape, 40)
    net.loss_grad(x, t, m)
    want = net.grads()
    y = net.forward(x).astype(np.float64)
    dy = (m * np.sin(y - t) / m.sum()).astype(np.float32)
    net.backward(x, dy)
    got = net.grads()
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()
    net.close()


def test_mlp_adam_step_matches_numpy():
    shape = (5, 16, 2, 4)
    net = learned.WarmStartMLP(*shape, seed=2)
    rng = np.random.default_rng(5)
    x, t, m = _data(rng, shape, 8)
    p = net.params().astype(np.float64)
    mm, vv = np.zeros_like(p), np.zeros_like(p)
    for step in range(1, 4):
        net.loss_grad(x, t, m)
        g = net.grads().astype(np.float64)
        net.adam_step(1e-2)
        mm = 0.9 * mm + 0.1 * g
        vv = 0.999 * vv + 0.001 * g * g
        p -= 1e-2 * (mm / (1 - 0.9 ** step)) / (np.sqrt(vv / (1 - 0.999 ** step)) + 1e-8)
        assert np.abs(net.params() - p).max() < 1e-5
    net.close()


def test_mlp_training_lowers_loss():
    shape = (46, 64, 2, 16)
    net = learned.WarmStartMLP(*shape, seed=4)
    rng = np.random.default_rng(9)
    x = rng.normal(0, 1, (256, 46)).astype(np.float32)
    w = rng.normal(0, 0.3, (46, 16))
    t = np.tanh(x @ w).astype(np.float32)  # a smooth target inside (-1, 1)
    m = np.ones_like(t)
    hist = net.fit(x, t, m, epochs=60, batch=64, lr=3e-3)
    assert hist[-1] < 0.1 * hist[0]
    net.close()


def test_mlp_rejects_bad_shapes():
    with pytest.raises(LogosQError) as e:
        learned.WarmStartMLP(0, 8, 1, 4)
    assert e.value.code == abi.LQ_ERR_INVALID_ARG
    net = learned.WarmStartMLP(4, 8, 1, 2)
    with pytest.raises(LogosQError) as e:
        net.set_params(np.zeros(net.num_params + 1, dtype=np.float32))
    assert e.value.code == abi.LQ_ERR_PARAM_COUNT
    net.close()


@pytest.mark.parametrize("n", [4, 6, 9, 12])
def test_lanczos_matches_eigvalsh(n):
    rec = workloads.heisenberg_instances(1, seed=20 + n, n_lo=n, n_hi=n)[0]
    terms = learned.chain_terms(rec)
    want = np.linalg.eigvalsh(oracle.dense_hamiltonian(n, terms))[0]
    got, iters = learned.lanczos_ground_energy(n, terms)
    assert abs(got - want) < 1e-10 * max(1.0, abs(want)), (got, want, iters)


def test_lanczos_bounds_variational_energy():
    """E0 at n = 16 lies below every ansatz energy (variational principle)."""
    n = 16
    rec = workloads.heisenberg_instances(1, seed=33, n_lo=n, n_hi=n)[0]
    terms = learned.chain_terms(rec)
    e0, _ = learned.lanczos_ground_energy(n, terms)
    _, E, _ = learned.batched_vqe([rec], [learned.fixed_start(n)], iters=40)
    assert e0 < E[0].min()


def test_lanczos_rejects_complex_hamiltonian():
    t = np.zeros(1, dtype=abi.TERM_DTYPE)
    t[0]["coefficient"] = 1.0
    t[0]["xmask"] = 1
    t[0]["zmask"] = 1
    t[0]["ny"] = 1
    with pytest.raises(LogosQError) as e:
        learned.lanczos_ground_energy(3, t)
    assert e.value.code == abi.LQ_ERR_UNSUPPORTED


def test_warm_start_beats_random_init():
    """Disordered XYZ chains, n 10-12.  Train on 768 chains: supervised on the
    optima of 100 batched VQE iterations from the fixed small-angle start
    (early stopping on a 10% held-out split), then 150 steps on the simulator's
    energy.  On 64 fresh chains the network's angles start much lower in
    energy than random angles and come within 0.1 of the best energy found in
    fewer VQE iterations."""
    train = workloads.disordered_chains(768, seed=5, n_lo=10, n_hi=12)
    X, T, M, _, _ = learned.optimum_dataset(train, iters=100)
    net = learned.WarmStartMLP(seed=1)
    hist = net.fit(X, T, M, epochs=100, batch=128, lr=1e-3, val_frac=0.1)
    assert hist[-1] < hist[0]
    eh = net.energy_train(train, 150, lr=3e-4)
    assert eh[-1] < eh[0]
    ev = workloads.disordered_chains(64, seed=6, n_lo=10, n_hi=12)
    rng = np.random.default_rng(6)
    iters = 150
    _, Ew, _ = learned.batched_vqe(ev, net.warm_start(ev), iters)
    _, Er, _ = learned.batched_vqe(ev, [learned.random_start(r["n"], rng) for r in ev], iters)
    best = np.minimum(Ew.min(axis=1), Er.min(axis=1))
    gw, gr = np.median(Ew[:, 0] - best), np.median(Er[:, 0] - best)
    assert gw < 0.7 * gr, (gw, gr)
    iw = learned.iterations_to(Ew, best, 0.1)
    ir = learned.iterations_to(Er, best, 0.1)
    assert np.median(iw) < np.median(ir), (np.median(iw), np.median(ir))
    net.close()
