"""Learned warm start: the MLP's GPU arithmetic against a torch float64
reference, training on the GPU, and the warm start in the corrector loop.
Both networks are checked: PSB_MLP_SILU6 (the configured 6 -> 64 -> 64 -> 1
SiLU network) and PSB_MLP_RELU7 (7 inputs, ReLU).

The reference computes in float64 with the GPU's storage rounding applied at
the same points: weights, inputs and hidden activations rounded to BF16
(round-to-nearest-even), the rounding's derivative taken as 1 (the GPU
back-propagates through the stored BF16 activations). In the backward pass
the GPU's tensor-core products take the BF16-rounded pre-activation
gradients dz1, dz2 as operands (for dW1, dW2 and for dz2 W2), while the bias
and output-layer gradients sum them in FP32; the reference rounds at the
same places (LinearBF). What remains:
  * ReLU is exact, so only FP32 accumulation differs: 99% of outputs within
    1e-4 of the output scale, all within 2e-2 (an FP32 pre-activation a few
    ulp from a BF16 rounding boundary rounds the other way and moves the
    output by one BF16 step of one unit);
  * SiLU uses the hardware tanh approximation (relative error below 2^-10),
    which moves an activation across a BF16 rounding boundary more often:
    every output must lie within the first-order effect of one BF16 step
    (2^-8 relative) in every hidden activation of both layers;
  * the loss gradient within 2e-3 of its norm (ReLU) and 4e-3 (SiLU, whose
    derivative also carries the tanh approximation).
"""
import numpy as np
import pytest

import oracle
import psb_project_b200 as P
from psb_project_b200 import runtime as R

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

ARCHS = [R.MLP_SILU6, R.MLP_RELU7]


def bf16(t):
    return t.to(torch.bfloat16).to(torch.float64)


class _RoundSTE(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x):
        return bf16(x)

    @staticmethod
    def backward(ctx, g):
        return g


class LinearBF(torch.autograd.Function):
    """inp @ W^T whose backward rounds the incoming gradient to BF16, as the
    GPU's tensor-core backward does for both dinp and dW."""

    @staticmethod
    def forward(ctx, inp, W):
        ctx.save_for_backward(inp, W)
        return inp @ W.T

    @staticmethod
    def backward(ctx, g):
        inp, W = ctx.saved_tensors
        gq = bf16(g)
        return gq @ W, gq.T @ inp


def act_of(arch):
    return torch.nn.functional.silu if arch == R.MLP_SILU6 else torch.nn.functional.relu


def torch_forward(w, X, arch):
    W1, b1, W2, b2, W3, b3 = [torch.tensor(a, dtype=torch.float64, requires_grad=True) for a in P.mlp_unpack(w)]
    params = [W1, b1, W2, b2, W3, b3]
    Wq = [_RoundSTE.apply(p) for p in params]
    act = act_of(arch)
    x = bf16(torch.tensor(X[:, :R.MLP_INPUTS[arch]], dtype=torch.float64))
    h1 = _RoundSTE.apply(act(LinearBF.apply(x, Wq[0]) + Wq[1]))
    h2 = _RoundSTE.apply(act(LinearBF.apply(h1, Wq[2]) + Wq[3]))
    y = h2 @ Wq[4] + Wq[5]
    return y, params, (h1, h2)


def sample_features(n, seed):
    rng = np.random.default_rng(seed)
    X = np.zeros((n, 7), np.float32)
    X[:, 0] = rng.uniform(0.3, 1.3, n)
    X[:, 1] = rng.normal(0, 1.0, n)
    X[:, 2] = rng.normal(0, 0.5, n)
    X[:, 3] = rng.uniform(0, 6, n)
    X[:, 4] = rng.uniform(0, 1, n)
    X[:, 5] = rng.uniform(0, 3, n)
    X[:, 6] = rng.uniform(0, 6, n)
    return X


def sim_for_mlp(arch):
    sim = P.Simulation(P.dam_break((8, 8, 8), 0.005, (0.2, 0.2, 0.2), 0.01))
    sim.mlp_set_arch(arch)
    return sim


def test_network_selection():
    with P.Simulation(P.dam_break((8, 8, 8), 0.005, (0.2, 0.2, 0.2), 0.01)) as sim:
        assert sim.mlp_info() == {"arch": R.MLP_SILU6, "n_inputs": 6, "n_params": 4673}
        sim.mlp_set_arch(R.MLP_RELU7)
        assert sim.mlp_info() == {"arch": R.MLP_RELU7, "n_inputs": 7, "n_params": 4737}
        with pytest.raises(ValueError):
            sim.mlp_set_weights(P.mlp_init_weights(0, R.MLP_SILU6))
        with pytest.raises(R.PsbError):
            sim.mlp_set_arch(5)


@pytest.mark.parametrize("arch", ARCHS)
def test_forward_matches_torch(arch):
    w = P.mlp_init_weights(3, arch)
    X = sample_features(4096, 1)
    with sim_for_mlp(arch) as sim:
        sim.mlp_set_weights(w)
        y = sim.mlp_forward(X).astype(np.float64)
    ref, _, (h1, h2) = torch_forward(w, X, arch)
    ref = ref.detach().numpy()
    scale = np.max(np.abs(ref))
    err = np.abs(y - ref)
    if arch == R.MLP_RELU7:
        assert np.quantile(err / scale, 0.99) < 1e-4
        assert (err / scale).max() < 2e-2
    else:
        # one BF16 step (2^-8 relative) in every activation of both layers,
        # propagated to first order (|SiLU'| <= 1.1)
        W1, b1, W2, b2, W3, b3 = [np.asarray(a, np.float64) for a in P.mlp_unpack(w)]
        h1n, h2n = np.abs(h1.detach().numpy()), np.abs(h2.detach().numpy())
        bound = (h2n @ np.abs(W3) + 1.1 * (h1n @ np.abs(W2).T) @ np.abs(W3)) * 2.0 ** -8 + 1e-5 * scale
        assert np.all(err <= bound), float(np.max(err / bound))
        assert np.quantile(err / scale, 0.99) < 3e-3


@pytest.mark.parametrize("arch", ARCHS)
def test_loss_gradient_matches_torch(arch):
    w = P.mlp_init_weights(5, arch)
    X = sample_features(2048, 2)
    T = (0.3 * X[:, 3] + 0.1 * X[:, 1] ** 2).astype(np.float32)
    with sim_for_mlp(arch) as sim:
        sim.mlp_set_weights(w)
        loss, g = sim.mlp_loss_grad(X, T)
    y, params, _ = torch_forward(w, X, arch)
    L = torch.mean((y - torch.tensor(T, dtype=torch.float64)) ** 2)
    L.backward()
    gref = np.concatenate([p.grad.numpy().ravel() for p in params])
    assert loss == pytest.approx(L.item(), rel=1e-3)
    tol = 2e-3 if arch == R.MLP_RELU7 else 4e-3
    assert np.linalg.norm(g - gref) / np.linalg.norm(gref) < tol


def test_loss_gradient_tail_tile():
    """A batch that leaves the last 64-sample tile partly empty: the absent
    samples contribute nothing (same gradient as the torch reference)."""
    arch = R.MLP_SILU6
    w = P.mlp_init_weights(6, arch)
    X = sample_features(100, 4)
    T = (0.2 * X[:, 0]).astype(np.float32)
    with sim_for_mlp(arch) as sim:
        sim.mlp_set_weights(w)
        loss, g = sim.mlp_loss_grad(X, T)
    y, params, _ = torch_forward(w, X, arch)
    L = torch.mean((y - torch.tensor(T, dtype=torch.float64)) ** 2)
    L.backward()
    gref = np.concatenate([p.grad.numpy().ravel() for p in params])
    assert loss == pytest.approx(L.item(), rel=1e-3)
    assert np.linalg.norm(g - gref) / np.linalg.norm(gref) < 4e-3


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


def test_training_is_reproducible():
    """The whole learned pipeline -- record plain-PCISPH rows, then train --
    run twice from the same state gives the same weights bit for bit: the
    simulation sums in list order, the minibatches are drawn from a seeded
    counter-based generator, and each block's gradient partials are added in
    block order (no floating-point atomics)."""
    sc = P.dam_break((24, 20, 16), 0.005, (0.5, 0.4, 0.3), 0.01, seed=11).replace(warm_start=P.WARM_PREVIOUS)
    pos = P.scene_positions(sc)
    runs = []
    for _ in range(2):
        with P.Simulation(sc) as sim:
            sim.upload(pos)
            sim.presolve(20)
            sim.mlp_collect(stride=4, capacity=1 << 18)
            sim.step(6)
            sim.mlp_set_weights(P.mlp_init_weights(0))
            loss = sim.mlp_train(200, 4096, 2e-3, seed=5)
            runs.append((loss, sim.mlp_get_weights()))
    assert runs[0][0] == runs[1][0]
    assert np.array_equal(runs[0][1], runs[1][1])


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


def mid_dam_state(seed=17, steps=30):
    """A dam break 30 steps in (previous-pressure start), as the GPU leaves it."""
    sc = P.dam_break((24, 20, 16), 0.005, (0.5, 0.4, 0.3), 0.01, seed=seed).replace(warm_start=P.WARM_PREVIOUS)
    with P.Simulation(sc) as sim:
        sim.upload(P.scene_positions(sc))
        sim.presolve(20)
        sim.step(steps)
        return sc, sim.download()


@pytest.mark.parametrize("arch", ARCHS)
def test_features_match_oracle(arch):
    """The warm start's inputs as the GPU computes them (FP32, inside the
    density pass at x) against the oracle's FP64 restatement (orc_features)
    on the same state. f0 (count / 32) is exact; f3 (p / p_scale) within
    1e-6 relative; f4 (wall distance / h) within 2e-5 (FP32 coordinates
    near 0.5 m carry 3e-8 m, 6e-6 h); the neighbour sums f1, f2, f5, f6
    within 3e-5 of their column's largest magnitude (~33 FP32 terms, and
    f1's density deviation is scaled by 100). The network reads the first
    n_in columns; the rest are 0."""
    sc, snap = mid_dam_state()
    with P.Simulation(sc.replace(warm_start=P.WARM_LEARNED)) as sim:
        sim.mlp_set_arch(arch)
        sim.mlp_set_weights(P.mlp_init_weights(1, arch))
        sim.upload(snap["pos"], snap["vel"], snap["vel_half"], snap["pressure"])
        F, _ = sim.warm_start()
        after = sim.download()
    ref = oracle.features(sc, snap["pos"], snap["vel"], snap["pressure"])
    n_in = R.MLP_INPUTS[arch]
    assert np.array_equal(after["pressure"], snap["pressure"])     # the carried pressure stays
    assert np.array_equal(F[:, 0], ref[:, 0].astype(np.float32))
    assert np.max(np.abs(F[:, 3] - ref[:, 3]) / np.maximum(np.abs(ref[:, 3]), 1e-30)) <= 1e-6
    assert np.max(np.abs(F[:, 4] - ref[:, 4])) <= 2e-5
    for k in [1, 2, 5] + ([6] if n_in == 7 else []):
        scale = np.max(np.abs(ref[:, k]))
        assert np.max(np.abs(F[:, k] - ref[:, k])) <= 3e-5 * scale, (k, np.max(np.abs(F[:, k] - ref[:, k])), scale)
    assert np.all(F[:, n_in:] == 0.0)


@pytest.mark.parametrize("arch", ARCHS)
def test_learned_step_matches_oracle(arch):
    """One learned-start step on the GPU against the oracle started from the
    same initial pressure. psb_warm_start returns the network's prediction
    p0 for the state (and leaves the state as it is); the oracle's config
    PCISPH step with the previous-pressure start from p0 is then the same
    method. The network is trained briefly on the GPU so that p0 is a
    realistic guess. The prediction p0 is compared with the oracle's network
    first; the step's tolerances are the config-PCISPH step's
    (test_gpu_parity): density 1e-5 element-wise, pressure and velocities
    1e-4 of their max."""
    sc, snap = mid_dam_state()
    with P.Simulation(sc) as gen:
        gen.mlp_set_arch(arch)
        gen.upload(snap["pos"], snap["vel"], snap["vel_half"], snap["pressure"])
        gen.mlp_collect(stride=2, capacity=1 << 18)
        gen.step(6)
        gen.mlp_collect(0)
        gen.mlp_set_weights(P.mlp_init_weights(2, arch))
        gen.mlp_train(300, 2048, 2e-3, seed=4)
        w = gen.mlp_get_weights()
    with P.Simulation(sc.replace(warm_start=P.WARM_LEARNED)) as sim:
        sim.mlp_set_arch(arch)
        sim.mlp_set_weights(w)
        sim.upload(snap["pos"], snap["vel"], snap["vel_half"], snap["pressure"])
        F, p0 = sim.warm_start()
        sim.step(1)
        out = sim.download()
        sg = sim.stats()
    assert np.all(p0 >= 0) and np.max(p0) > 0
    # the prediction itself: the oracle's network on the GPU's own inputs
    # (the network arithmetic, the forward test's 99th-percentile bound) and
    # on the oracle's FP64 inputs (the whole learned path; an input that
    # differs by its 3e-5 tolerance can round to the neighbouring BF16 value)
    n_in, act = R.MLP_INPUTS[arch], ("silu" if arch == R.MLP_SILU6 else "relu")
    p_scale = sc.rho0 * float(np.linalg.norm(sc.gravity)) * 0.1
    y, _, _ = oracle.mlp_forward(w, F, n_in, act)
    ref_own = np.maximum(0.0, y) * p_scale
    scale = float(np.max(ref_own))
    assert np.quantile(np.abs(p0 - ref_own), 0.99) <= 3e-3 * scale
    ref_full = oracle.learned_pressure(sc, snap["pos"], snap["vel"], snap["pressure"], w, arch)
    d = np.abs(p0 - ref_full)
    assert np.median(d) <= 1e-3 * scale and np.quantile(d, 0.99) <= 2e-2 * scale, (np.median(d), np.quantile(d, 0.99), scale)
    orc = oracle.OracleSim(sc, snap["pos"], snap["vel"], snap["vel_half"], p0, float_state=True)
    so = orc.step()
    for k in range(min(so.iters, sg.iters) + 1):
        assert abs(sg.err[k] - so.err[k]) <= 1e-5, (k, sg.err[k], so.err[k])
    if sg.iters != so.iters:
        k = min(sg.iters, so.iters)
        assert abs(so.err[k] - sc.eta) <= 2e-6
        return
    assert np.max(np.abs(out["density"] - orc.rho) / orc.rho) <= 1e-5
    scale = max(np.max(np.abs(orc.p)), 1e-30)
    assert np.max(np.abs(out["pressure"] - orc.p)) <= 1e-4 * scale
    assert np.max(np.abs(out["vel_half"] - orc.vel_half)) <= 1e-4 * np.max(np.abs(orc.vel_half))
