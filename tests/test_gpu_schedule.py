"""The learned schedule: the network's CUDA forward and backward kernels against the CPU
restatement (oracle/sched_oracle.py), training on the device, and the schedule's two promises:
results identical to the fixed heuristics, and what the trained network gains over them."""
import os

import numpy as np
import pytest

import sched_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small(pkg):
    g = pkg.graphs.rmat(10, seed=2)
    d = pkg.DeviceGraph.from_graph(g)
    yield d
    d.close()


def test_forward_and_gradient_match_cpu(small):
    rng = np.random.default_rng(0)
    p = (0.3 * rng.standard_normal(sched_oracle.NP)).astype(np.float32)
    x = rng.standard_normal((333, 8)).astype(np.float32)
    y = rng.integers(0, 8, 333).astype(np.int32)
    small.sched_set_weights(p)
    z = small.sched_forward(x)
    zr, _ = sched_oracle.forward(p, x)
    np.testing.assert_allclose(z, zr, rtol=1e-4, atol=1e-5)
    grad, loss = small.sched_grad(x, y)
    lr, gr = sched_oracle.loss_and_grad(p, x, y)
    assert abs(loss - lr) < 1e-4 * max(1.0, abs(lr))
    np.testing.assert_allclose(grad, gr, rtol=2e-3, atol=2e-6)
    # finite differences on a few parameters
    for i in (0, 17, 260, 300, 551):
        e = np.zeros_like(p, dtype=np.float64)
        e[i] = 1e-3
        fd = (sched_oracle.loss_and_grad(p + e, x, y)[0] - sched_oracle.loss_and_grad(p - e, x, y)[0]) / 2e-3
        assert abs(fd - grad[i]) < 2e-3 * max(1.0, abs(fd)), (i, fd, grad[i])


def test_training_lowers_the_loss(small):
    rng = np.random.default_rng(1)
    x = rng.standard_normal((512, 8)).astype(np.float32)
    y = (x[:, 0] > 0).astype(np.int32) + 2 * (x[:, 1] > 0.5).astype(np.int32)
    # (small random weights: with all-zero weights the hidden layer has no gradient)
    small.sched_set_weights((0.1 * rng.standard_normal(sched_oracle.NP)).astype(np.float32))
    l0 = small.sched_grad(x, y)[1]
    l1 = small.sched_train(x, y, steps=500, lr=0.5)
    assert l1 < 0.5 * l0
    pred = np.argmax(small.sched_forward(x), 1)
    assert (pred == y).mean() > 0.9


WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "graph-intermedia-representation_b200", "schedule_weights.npy")


@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="no trained schedule weights committed")
def test_learned_schedule_is_exact_and_gains(pkg, orc):
    """Same levels and distances under the learned schedule; and on the high-diameter lattice
    (large weights) its bucket width beats the reference's fixed Delta = 16 (CUDA-event medians of
    five calls each)."""
    import torch
    lat = pkg.graphs.lattice(side=200, seed=43)
    d = pkg.DeviceGraph.from_graph(lat)
    src = torch.from_numpy(pkg.graphs.sources_with_edges(lat, 8, 3)).to("cuda:0")
    out_f = torch.empty((8, lat.V), dtype=torch.int64, device="cuda:0")
    out_l = torch.empty_like(out_f)
    def median_ms(fn, reps=5):
        fn()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts)) * 1e-3

    t_fixed = median_ms(lambda: d.sssp(src, delta=16, weights=pkg.native.WEIGHT_STORED, out=out_f))
    d.use_learned_schedule(WEIGHTS)
    t_learned = median_ms(lambda: d.sssp(src, delta=0, weights=pkg.native.WEIGHT_STORED, out=out_l))
    x, cls = d.sched_trace()
    assert torch.equal(out_f, out_l)
    fb, fa = orc.normalize(lat.V, lat.fw_beg, lat.fw_adj)
    np.testing.assert_array_equal(out_l[0].cpu().numpy().astype(np.uint64),
                                  orc.sssp(lat.V, fb, fa, [int(src[0])], w=lat.w))
    chosen = int(pkg.DeviceGraph.delta_choices()[cls[0] - 2])
    print(f"lattice 200^2 SSSP x8: fixed delta 16 {1e3 * t_fixed:.1f} ms, learned delta {chosen} "
          f"{1e3 * t_learned:.1f} ms, gain {t_fixed / t_learned:.2f}x")
    assert chosen > 16
    assert t_learned < t_fixed
    # BFS directions from the network: identical levels
    lv_l = d.bfs(src)
    d.set_schedule(pkg.native.SCHEDULE_FIXED)
    lv_f = d.bfs(src)
    np.testing.assert_array_equal(torch.as_tensor(lv_l).numpy() if hasattr(lv_l, "numpy") else lv_l, lv_f)
    d.close()
