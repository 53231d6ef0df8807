"""The learned cost model: its FP32 GPU gradient against an FP64 CPU oracle of the same
network, training, and how well the trained model alone ranks the candidate plans of a
held-out circuit (measured device time of its pick against every candidate's, identical
amplitudes)."""
import numpy as np
import pytest
import torch

import litequantumcomputingsimulator_b200 as lq
from litequantumcomputingsimulator_b200 import costmodel as CM
from litequantumcomputingsimulator_b200 import workloads as W

pytestmark = pytest.mark.gpu
F, H = CM.FEATURES, 64


def unpack(w):
    w = w.astype(np.float64)
    i = 0
    W1 = w[i:i + H * F].reshape(H, F); i += H * F
    b1 = w[i:i + H]; i += H
    W2 = w[i:i + H * H].reshape(H, H); i += H * H
    b2 = w[i:i + H]; i += H
    W3 = w[i:i + H]; i += H
    b3 = w[i]
    return W1, b1, W2, b2, W3, b3


def oracle_loss_grad(w, x, y):
    """FP64 restatement: two ReLU layers of 64, linear output, mean squared error."""
    W1, b1, W2, b2, W3, b3 = unpack(w)
    x = x.astype(np.float64)
    a1 = x @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    out = h2 @ W3 + b3
    n = len(y)
    d = 2 * (out - y) / n
    g2 = (d[:, None] * W3[None, :]) * (a2 > 0)
    g1 = (g2 @ W2) * (a1 > 0)
    grads = [g1.T @ x, g1.sum(0), g2.T @ h1, g2.sum(0), d @ h2, np.array([d.sum()])]
    return float(np.mean((out - y) ** 2)), np.concatenate([g.reshape(-1) for g in grads])


def test_gradient_matches_fp64_oracle():
    rng = np.random.default_rng(0)
    n_params = H * F + H + H * H + H + H + 1
    w = (rng.standard_normal(n_params) * 0.2).astype(np.float32)
    CM.set_weights(w)
    x = rng.uniform(0, 1, (96, F)).astype(np.float32)
    y = rng.standard_normal(96).astype(np.float32)
    loss, g = CM.gradient(x, y)
    loss_o, g_o = oracle_loss_grad(w, x, y)
    assert abs(loss - loss_o) <= 1e-4 * max(1.0, abs(loss_o))
    scale = np.max(np.abs(g_o))
    assert np.max(np.abs(g - g_o)) <= 2e-4 * scale
    CM.clear()


def test_training_fits_a_smooth_function():
    rng = np.random.default_rng(1)
    x = rng.uniform(0, 1, (2000, F)).astype(np.float32)
    y = (np.sin(3 * x[:, 0]) + x[:, 1] * x[:, 2] - 0.5 * x[:, 4]).astype(np.float32)
    loss = CM.train(x, y, epochs=1500, lr=3e-3, seed=2)
    assert loss < 0.05 * float(np.var(y))
    pred = CM.predict(x[:10])
    assert np.max(np.abs(pred - y[:10])) < 0.5
    CM.clear()


def _time_ms(prog, sv, reps=5):
    prog.apply(sv)
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times = []
    for _ in range(reps):
        s.record()
        prog.apply(sv)
        e.record()
        torch.cuda.synchronize()
        times.append(s.elapsed_time(e))
    return float(np.median(times))


def _candidate_times(circuit, init):
    """Measured device time of every candidate plan the learned mode chooses among."""
    out = {}
    for name, prog in CM.candidate_programs(circuit):
        sv = lq.Statevector.from_numpy(init)
        out[name] = _time_ms(prog, sv, reps=3)
    return out


def test_learned_plan_ranking(monkeypatch):
    """Trained on the engine's own timings of five random-mix circuits, the model alone
    (LQCS_LEARNED_JUDGE=1: no candidate is timed) must pick, for a held-out circuit, a plan
    within 15 % of the fastest candidate and faster than the greedy plan, with amplitudes
    equal to the greedy plan's.  It is not required to beat the default plan (register tile
    passes of 2^12 amplitudes): on these circuits the default is the fastest candidate or
    within a few percent of it, so the model's value is choosing without timing candidates
    (what the autotuner does), not a faster plan than the default."""
    train_set = [W.random_mix_circuit(n, d, seed) for n, d, seed in
                 [(19, 12, 1), (20, 16, 2), (21, 10, 3), (20, 20, 4), (21, 14, 5)]]
    x, y = CM.collect(train_set)
    loss = CM.train(x, y, epochs=3000, lr=3e-3, seed=0)
    assert loss < 0.5 * float(np.var(y))
    held = W.random_mix_circuit(21, 24, seed=99)
    init = W.gaussian_state(21, seed=7)
    monkeypatch.setenv("LQCS_LEARNED_JUDGE", "1")
    greedy = lq.simulator.CompiledCircuit(held, True, 0, CM.GREEDY)
    learned = lq.simulator.CompiledCircuit(held, True, 0, CM.LEARNED)
    outs = []
    for prog in (greedy, learned):
        sv = lq.Statevector.from_numpy(init)
        prog.apply(sv)
        outs.append(sv.to_numpy())
    assert np.max(np.abs(outs[0] - outs[1])) < 1e-12
    times = _candidate_times(held, init)
    sv = lq.Statevector.from_numpy(init)
    t_learned = _time_ms(learned, sv)
    t_greedy = _time_ms(greedy, sv)
    best = min(times.values())
    assert t_learned <= 1.15 * best, (t_learned, times)
    assert t_learned < t_greedy, (t_learned, t_greedy)
    CM.clear()
    fallback = lq.simulator.CompiledCircuit(held, True, 0, CM.LEARNED)
    assert fallback.n_ops == greedy.n_ops
