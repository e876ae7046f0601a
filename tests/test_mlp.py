"""Learned warm start: the MLP's GPU arithmetic against a torch float64
reference, training on the GPU, and the warm start in the corrector loop.

The reference computes in float64 with the GPU's storage rounding applied at
the same points: weights, inputs and hidden activations rounded to BF16
(round-to-nearest-even), the rounding's derivative taken as 1 (the GPU
back-propagates through the stored BF16 activations). The activation is
ReLU, exact in both; what remains is FP32 accumulation against float64:
  * forward: 99% of outputs within 1e-4 of the output scale, all within 2e-2
    (an FP32 pre-activation a few ulp from a BF16 rounding boundary rounds
    the other way and moves the output by one BF16 step of one unit);
  * loss gradient: within 2e-3 of its norm.
"""
import numpy as np
import pytest

import psb_project_b200 as P
from psb_project_b200 import runtime as R

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def bf16(t):
    return t.to(torch.bfloat16).to(torch.float64)


class _RoundSTE(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x):
        return bf16(x)

    @staticmethod
    def backward(ctx, g):
        return g


def torch_forward(w, X):
    W1, b1, W2, b2, W3, b3 = [torch.tensor(a, dtype=torch.float64, requires_grad=True) for a in P.mlp_unpack(w)]
    params = [W1, b1, W2, b2, W3, b3]
    Wq = [_RoundSTE.apply(p) for p in params]
    x = bf16(torch.tensor(X[:, :R.MLP_IN], dtype=torch.float64))
    h1 = _RoundSTE.apply(torch.nn.functional.relu(x @ Wq[0].T + Wq[1]))
    h2 = _RoundSTE.apply(torch.nn.functional.relu(h1 @ Wq[2].T + Wq[3]))
    y = h2 @ Wq[4] + Wq[5]
    return y, params


def sample_features(n, seed):
    rng = np.random.default_rng(seed)
    X = np.zeros((n, R.MLP_IN), np.float32)
    X[:, 0] = rng.uniform(0.3, 1.3, n)
    X[:, 1] = rng.normal(0, 1.0, n)
    X[:, 2] = rng.normal(0, 0.5, n)
    X[:, 3] = rng.uniform(0, 6, n)
    X[:, 4] = rng.uniform(0, 1, n)
    X[:, 5] = rng.uniform(0, 3, n)
    X[:, 6] = rng.uniform(0, 6, n)
    return X


def sim_for_mlp():
    return P.Simulation(P.dam_break((8, 8, 8), 0.005, (0.2, 0.2, 0.2), 0.01))


def test_forward_matches_torch():
    w = P.mlp_init_weights(3)
    X = sample_features(4096, 1)
    with sim_for_mlp() as sim:
        sim.mlp_set_weights(w)
        y = sim.mlp_forward(X).astype(np.float64)
    ref, _ = torch_forward(w, X)
    ref = ref.detach().numpy()
    scale = np.max(np.abs(ref))
    err = np.abs(y - ref) / scale
    assert np.quantile(err, 0.99) < 1e-4
    assert err.max() < 2e-2


def test_loss_gradient_matches_torch():
    w = P.mlp_init_weights(5)
    X = sample_features(2048, 2)
    T = (0.3 * X[:, 3] + 0.1 * X[:, 1] ** 2).astype(np.float32)
    with sim_for_mlp() as sim:
        sim.mlp_set_weights(w)
        loss, g = sim.mlp_loss_grad(X, T)
    y, params = torch_forward(w, X)
    L = torch.mean((y - torch.tensor(T, dtype=torch.float64)) ** 2)
    L.backward()
    gref = np.concatenate([p.grad.numpy().ravel() for p in params])
    assert loss == pytest.approx(L.item(), rel=1e-3)
    assert np.linalg.norm(g - gref) / np.linalg.norm(gref) < 2e-3


def test_training_reduces_loss_on_a_known_function():
    """Record (features, converged pressure) rows from a small dam break and
    train on them: the GPU's Adam loop must cut the loss five-fold."""
    sc = P.dam_break((24, 20, 16), 0.005, (0.5, 0.4, 0.3), 0.01, seed=11).replace(warm_start=P.WARM_PREVIOUS)
    with P.Simulation(sc) as sim:
        sim.upload(P.scene_positions(sc))
        sim.presolve(20)
        sim.mlp_collect(stride=4, capacity=1 << 18)
        sim.step(8)
        rows, X, T = sim.mlp_dataset()
        assert rows > 0 and np.isfinite(X).all() and np.isfinite(T).all()
        sim.mlp_set_weights(P.mlp_init_weights(0))
        first = sim.mlp_train(1, 1024, 1e-3, seed=1)
        last = sim.mlp_train(600, 1024, 2e-3, seed=2)
    assert last < 0.2 * first


def test_learned_warm_start_beats_plain():
    """Collect (features, converged pressure) pairs from warm-started steps,
    train, then run the same steps learned and plain: the learned start must
    need fewer corrections at the same eta, and every step must converge."""
    base = P.dam_break((32, 32, 16), 0.005, (0.6, 0.4, 0.2), 0.01, seed=13)
    pos = P.scene_positions(base)
    with P.Simulation(base.replace(warm_start=P.WARM_PREVIOUS)) as sim:
        sim.upload(pos)
        sim.presolve(40)
        sim.mlp_collect(stride=2, capacity=1 << 20)
        sim.step(30)
        snap = sim.download()
        sim.mlp_set_weights(P.mlp_init_weights(0))
        sim.mlp_train(1500, 4096, 2e-3, seed=3)
        w = sim.mlp_get_weights()
    iters = {}
    for name, mode in (("learned", P.WARM_LEARNED), ("plain", P.WARM_ZERO)):
        with P.Simulation(base.replace(warm_start=mode)) as sim:
            if mode == P.WARM_LEARNED:
                sim.mlp_set_weights(w)
            sim.upload(snap["pos"], snap["vel"], snap["vel_half"], snap["pressure"])
            its = []
            for _ in range(10):
                sim.step(1)
                st = sim.stats()
                its.append(st.iters)
                assert st.converged == 1
                assert st.err[st.iters] <= base.eta
            iters[name] = np.mean(its)
    assert iters["learned"] < iters["plain"], iters
