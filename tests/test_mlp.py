"""The learned starting iterate: its network's forward pass and gradient on the
tensor cores against the numpy restatement (oracle/mlp_oracle.py), the
restatement's gradient against finite differences, training, and what the
trained network changes in the ionisation solve of an HII-region run.
"""
import os
import sys

import numpy as np
import pytest

import common  # noqa: F401  (puts the repo root on sys.path)

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_oracle  # noqa: E402

import torch_b200  # noqa: E402
from torch_b200 import workloads  # noqa: E402


def random_params(seed, normalise=True):
    rng = np.random.default_rng(seed)
    p = torch_b200.mlp_init_params(seed)
    n = torch_b200.MLP_NTRAIN
    p[:n] += rng.normal(0, 0.05, n).astype(np.float32)  # non-zero biases too
    if normalise:
        p[n:n + 5] = rng.normal(0, 1, 5)
        p[n + 5:n + 10] = rng.uniform(0.5, 2.0, 5)
        p[n + 10:n + 13] = rng.normal(0, 1, 3)
        p[n + 13:n + 16] = rng.uniform(0.5, 2.0, 3)
    return p


def random_records(seed, n):
    rng = np.random.default_rng(seed)
    r = rng.normal(0, 1.5, (n, 8)).astype(np.float32)
    return r


def test_oracle_gradient_matches_finite_differences():
    p = random_params(1).astype(np.float64)
    rec = random_records(2, 64).astype(np.float64)
    w = np.array([1.0, 0.5, 0.25])
    g, _ = mlp_oracle.gradient(p, rec, w, emulate=False)
    rng = np.random.default_rng(3)
    idx = rng.choice(mlp_oracle.NTRAIN, 60, replace=False)
    eps = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (mlp_oracle.gradient(pp, rec, w, emulate=False)[1] - mlp_oracle.gradient(pm, rec, w, emulate=False)[1]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.01171875, -3.0, 1e-30, 65504.0], dtype=np.float32)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even mantissa is 1.0;
    # 1 + 3*2^-8 is a tie between 1 + 2^-7 and 1 + 2^-6: even is 1 + 2^-6
    want = np.array([1.0, 1.0, 1.015625, -3.0, 1e-30, 65536.0], dtype=np.float32)
    got = mlp_oracle.bf16(x)
    assert got[0] == want[0] and got[1] == want[1] and got[2] == want[2] and got[3] == want[3]
    assert abs(got[4] - 1e-30) / 1e-30 < 4e-3 and got[5] == want[5]


@pytest.mark.gpu
def test_forward_matches_oracle():
    p = random_params(5)
    x = random_records(6, 1000)[:, :5]
    m = torch_b200.Mlp(p)
    y = m.forward(x)
    m.close()
    ref = mlp_oracle.forward(p, x)
    err = np.abs(y - ref) / (np.abs(ref) + 1.0)
    print(f"forward: median {np.median(err):.2e} max {err.max():.2e}")
    assert np.median(err) < 1e-5 and err.max() < 2e-2


@pytest.mark.gpu
def test_gradient_matches_oracle():
    p = random_params(7)
    rec = random_records(8, 1000)
    w = np.array([1.0, 0.5, 0.25], dtype=np.float32)
    m = torch_b200.Mlp(p)
    g, loss = m.gradient(rec, w)
    m.close()
    gr, lr = mlp_oracle.gradient(p, rec, w)
    assert abs(loss - lr) <= 1e-4 * abs(lr)
    o = 0
    for name, n in (("W1", 320), ("b1", 64), ("W2", 4096), ("b2", 64), ("W3", 192), ("b3", 3)):
        a, b = g[o:o + n].astype(np.float64), gr[o:o + n]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        print(f"grad {name}: rel {rel:.2e}")
        assert rel <= 1e-2, name
        o += n


@pytest.mark.gpu
def test_training_reduces_loss():
    rng = np.random.default_rng(9)
    x = rng.uniform(-2, 2, (20000, 5)).astype(np.float32)
    t = np.stack([np.tanh(x[:, 0] * x[:, 1]), np.sin(x[:, 2]) + 0.5 * x[:, 3], x[:, 4] ** 2 / 4], 1)
    rec = np.concatenate([x, t], 1).astype(np.float32)
    m = torch_b200.Mlp(seed=1)
    hist = m.train(rec, epochs=30, batch=2048, lr=3e-3, seed=2, out_weight=(1, 1, 1))
    y = m.forward(x[:2000])
    m.close()
    print("loss", hist[0], hist[-1])
    assert hist[-1] < 0.1 * hist[0]
    assert np.mean((y - t[:2000]) ** 2) < 0.05


def tolerance_probe_params(delta=4.342727686266e-4):
    """A network whose output is constant: every front cell is predicted slow
    and starts at odds (1 + 1e-3) times those of the plain start, one solver
    tolerance away.  The state change this causes is the scale against which
    the learned start's change is compared."""
    p = np.zeros(torch_b200.MLP_NPARAMS, dtype=np.float32)
    n = torch_b200.MLP_NTRAIN
    p[n - 3:n] = (delta, 0.0, 2.0)
    p[n + 5:n + 10] = 1.0
    p[n + 13:n + 16] = 1.0
    return p


def ifront_x(hii, n):
    """I-front distance (cells) from the central star along +x: first cell
    with HII < 0.5, linearly interpolated (scripts/misc/calc_if.py:43-56)."""
    x = hii.reshape(n, n, n)[n // 2, n // 2, n // 2:]
    for i in range(1, len(x)):
        if x[i] < 0.5:
            return (i - 1) + (x[i - 1] - 0.5) / (x[i - 1] - x[i])
    return float(len(x))


@pytest.mark.gpu
def test_learned_start_on_hii_region():
    """Harvest front-cell solves from the plain method, train on the GPU, then
    run the same steps with the learned start: before each sweep the network
    runs once over the candidate front cells (chosen from the previous
    sweep's optical depths) and serves those it predicts to be slow; beside
    the plain first Picard iteration a served cell runs one from the
    prediction, which is accepted when it passes the convergence test and the
    plain one does not.  Reports the iterations per front cell with and
    without the network and how far each moves the state from the plain run,
    beside a start one solver tolerance off; the I-front stays within 0.5
    cell."""
    n, steps = 32, 40
    tp, ic = workloads.hii_region(n=n, seed=4)
    plain = torch_b200.Torch(tp, ic)
    plain.harvest(1 << 20)
    plain.stats_enable(True)
    plain.run_steps(steps)
    rec, total = plain.harvest_read()
    st_plain = plain.stats()
    s_plain = plain.state()
    plain.close()
    print("records", total, "front cells", st_plain["front_cells"], "front iters", st_plain["front_iters"])
    assert total > 1000
    m = torch_b200.Mlp(seed=3)
    hist = m.train(rec, epochs=40, batch=1024, lr=2e-3, seed=5)
    print("training loss", hist[0], hist[-1])
    assert hist[-1] < 0.5 * hist[0]

    def run_with(net):
        r = torch_b200.Torch(tp, ic)
        r.learned_start(net)
        r.stats_enable(True)
        r.run_steps(steps)
        out = (r.stats(), r.state())
        r.close()
        return out

    st, s = run_with(m)
    m.close()
    probe = torch_b200.Mlp(tolerance_probe_params())
    st_tol, s_tol = run_with(probe)
    probe.close()
    acc = st["learned_accepted"] / max(1, st["learned_cells"])
    it_plain = st_plain["front_iters"] / max(1, st_plain["front_cells"])
    it_learned = st["front_iters"] / max(1, st["front_cells"])
    print(f"learned cells {st['learned_cells']} accepted {acc:.3f}; front iterations per cell: plain {it_plain:.3f} "
          f"learned {it_learned:.3f}")
    assert 0 < st["learned_cells"] <= st["front_cells"]
    # the candidates are chosen before each sweep from the previous sweep's
    # optical depths: the probe network (every candidate predicted slow)
    # serves most of the front cells the sweep finds
    assert 0.5 * st_tol["front_cells"] <= st_tol["learned_cells"] <= st_tol["front_cells"]
    dev = {k: common.rel_l1(s.U[i], s_plain.U[i]) for k, i in (("den", 0), ("E", 1), ("hii", 2))}
    tol = {k: common.rel_l1(s_tol.U[i], s_plain.U[i]) for k, i in (("den", 0), ("E", 1), ("hii", 2))}
    print("state vs plain after", steps, "steps, learned:", {k: f"{v:.2e}" for k, v in dev.items()},
          "one-tolerance start:", {k: f"{v:.2e}" for k, v in tol.items()})
    r_plain, r_learned = ifront_x(s_plain.Q[2], n), ifront_x(s.Q[2], n)
    print(f"I-front: plain {r_plain:.3f} learned {r_learned:.3f} cells")
    assert abs(r_plain - r_learned) <= 0.5
    assert dev["den"] <= 1e-3 and dev["E"] <= 1e-2


@pytest.mark.gpu
def test_learned_start_gain_after_training_at_scale():
    """The gain the trained network gives on the 256^3 HII region (lognormal
    cloud, seed 12345, 2 pc box), FP32 form: the plain solve records front-cell
    solves in 10-step blocks until 10^7 records (or 400 steps), the network
    trains on them on the GPU (30 epochs), then the same 8 steps run from the
    same saved state with and without it.  The network must cut the Picard
    iterations per front cell (its prediction is tried beside the plain first
    iteration, so a rejected one costs no iteration), and the I-front and the
    state stay with the plain run's.  (On the same cloud at 128^3, cells twice
    as large, the plain solve already needs fewer iterations and the network
    gains little.)"""
    n = 256
    tp, ic = workloads.hii_region(n=n, seed=12345)
    t = torch_b200.Torch(tp, ic, precision=torch_b200.PRECISION_FP32)
    t.harvest(10_000_000)
    steps = 0
    while steps < 400 and t.harvest_read(count_only=True) < 10_000_000:
        t.run_steps(10)
        steps += 10
    rec, total = t.harvest_read()
    t.harvest(0)
    blob = t.checkpoint()
    print("records", total, "harvest steps", steps)
    assert total > 1_000_000
    m = torch_b200.Mlp(seed=11)
    hist = m.train(rec, epochs=30, batch=8192, lr=2e-3, seed=12)
    del rec
    print("training loss", hist[0], hist[-1])
    runs = {}
    for name, net in (("plain", None), ("learned", m)):
        t.restore(blob)
        t.learned_start(net)
        t.stats_enable(True)
        t.run_steps(8)
        runs[name] = (t.stats(reset=True), t.state())
        t.stats_enable(False)
    t.learned_start(None)
    t.close()
    m.close()
    st_p, s_p = runs["plain"]
    st_l, s_l = runs["learned"]
    it_p = st_p["front_iters"] / max(1, st_p["front_cells"])
    it_l = st_l["front_iters"] / max(1, st_l["front_cells"])
    acc = st_l["learned_accepted"] / max(1, st_l["learned_cells"])
    print(f"front cells {st_p['front_cells']}: Picard iterations per front cell plain {it_p:.3f}, learned {it_l:.3f}; "
          f"predictions accepted {acc:.3f} of {st_l['learned_cells']}")
    assert st_l["learned_cells"] > 0
    assert it_l < it_p
    fp, fl = common.ifront_cells(s_p.Q[2], n), common.ifront_cells(s_l.Q[2], n)
    print(f"I-front plain {fp:.4f} learned {fl:.4f} cells; density L1 {common.rel_l1(s_l.U[0], s_p.U[0]):.2e}")
    assert abs(fp - fl) <= 0.5
    assert common.rel_l1(s_l.U[0], s_p.U[0]) <= 1e-4
