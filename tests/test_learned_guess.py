"""The learned initial guess of the rate-and-state Newton solve, on the GPU.

* the training kernels' forward pass and gradient match the NumPy oracle (which is itself
  checked against finite differences in test_mlp_oracle.py), and so do the node kernel's
  two inference paths (per-thread, and warp-wide on the tensor cores);
* training on samples the plain solver records lowers the loss;
* on rate-and-state rough-fault runs (a narrow fault whose warps are all partly outside
  the rupture area, and a wider one with whole warps of live nodes, where the tensor-core
  network runs), most learned guesses pass the residual test, the accepted roots equal the
  plain solve's (judge mode), the slip differs from the plain run by rounding only, both
  runs have the same error against the FP64 oracle, and the learned guess needs fewer
  Newton iterations.
"""
import numpy as np
import pytest

import cases
import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def rand_net(seed=0):
    import dynfd3dcuda_b200 as dfd

    rng = np.random.default_rng(seed)
    w = dfd.mlp_init(seed, [40.0, -3.0, -2.0, 0.015], [10.0, 2.0, 1.5, 0.003], -0.5, 0.8)
    w[:dfd.MLP_TRAINABLE] += rng.normal(0, 0.05, dfd.MLP_TRAINABLE).astype(np.float32)
    x = np.stack([rng.uniform(20, 60, 3000), rng.uniform(-8, 1, 3000), rng.uniform(-4, 0, 3000),
                  rng.uniform(0.01, 0.02, 3000)], 1).astype(np.float32)
    y = rng.normal(-0.5, 0.8, 3000).astype(np.float32)
    return w, x, y


def test_forward_and_gradient_match_oracle():
    import dynfd3dcuda_b200 as dfd

    w, x, y = rand_net(1)
    yp = dfd.mlp_forward(w, x)
    ref = mo.predict(w, x)
    assert np.abs(yp - ref).max() < 1e-4 * (1 + np.abs(ref).max())
    loss, g = dfd.mlp_loss_grad(w, x, y)
    lref, gref = mo.loss_grad(w, x, y)
    assert abs(loss - lref) < 1e-5 * abs(lref)
    # FP32 accumulation over 3000 samples against FP64: relative to the gradient's scale
    assert np.abs(g - gref).max() < 2e-4 * np.abs(gref).max()


def test_node_inference_matches_oracle():
    """The node kernel's inference: per-thread network (hardware tanh) and tensor-core
    network (FP16 operands of the hidden layer), against the FP64 oracle; both errors are
    far below what the residual test and one Newton correction absorb."""
    import dynfd3dcuda_b200 as dfd

    w, x, _ = rand_net(3)
    ref = mo.predict(w, x)
    scale = 1.0 + np.abs(ref).max()
    y0 = dfd.mlp_forward_node(w, x, tensor_cores=False)
    y1 = dfd.mlp_forward_node(w, x, tensor_cores=True)
    e0 = np.abs(y0 - ref).max() / scale
    e1 = np.abs(y1 - ref).max() / scale
    print(f"per-thread {e0:.2e}, tensor cores {e1:.2e}")
    assert e0 < 5e-3 and e1 < 5e-3, (e0, e1)
    # an odd batch: the padding rows must not disturb the real ones
    y2 = dfd.mlp_forward_node(w, x[:1000 - 7], tensor_cores=True)
    assert np.array_equal(y2, y1[:1000 - 7])


def test_training_lowers_loss():
    import dynfd3dcuda_b200 as dfd

    rng = np.random.default_rng(5)
    x = np.stack([rng.uniform(20, 60, 20000), rng.uniform(-8, 1, 20000), rng.uniform(-4, 0, 20000),
                  rng.uniform(0.01, 0.02, 20000)], 1).astype(np.float32)
    y = (np.tanh(0.05 * (x[:, 0] - 40)) - 0.3 * x[:, 1] + 0.2 * x[:, 2]).astype(np.float32)
    w, hist = dfd.train_guess_net(np.column_stack([x, y]), epochs=20, batch=1024, lr=3e-3, seed=2)
    assert hist[-1] < 0.05 * hist[0]
    yp = dfd.mlp_forward(w, x)
    assert np.sqrt(np.mean((yp - y) ** 2)) < 0.1 * y.std()


def run(job, fx, st, steps, net=None):
    import dynfd3dcuda_b200 as dfd

    sim = dfd.Simulation(job, fx, st, None)
    if net is not None:
        sim.set_guess_net(net)
        sim.rs_profile(timing=False, judge=True)
    sim.run(0, steps)
    sim.synchronize()
    its, capped = sim.newton_stats()
    stats = sim.rs_solve_stats()
    out = {k: sim.fault(k).astype(np.float64) for k in ("slip", "Vs1", "State")}
    sim.close()
    return out, its, capped, stats


@pytest.mark.parametrize("ny", [76, 128])
def test_learned_guess_same_roots_fewer_iterations(oracle_lib, ny):
    import dynfd3dcuda_b200 as dfd

    # training data: plain solver on another seed of the same configuration
    pt, fxt, stt, _, _, meta = cases.rs_rough_case(ny, 24, 40, seed=41, L=0.02, steps=60)
    sim = dfd.Simulation(pt, fxt, stt, None)
    sim.newton_record(400000, 1)
    sim.run(0, meta["steps"])
    samples = sim.newton_samples(400000)
    sim.close()
    assert len(samples) > 10000
    w, hist = dfd.train_guess_net(samples, epochs=60, batch=1024, lr=3e-3, seed=4)
    assert hist[-1] < hist[0]

    p, fx, st, _, _, meta = cases.rs_rough_case(ny, 24, 40, seed=31, L=0.02, steps=60)
    steps = meta["steps"]
    plain, its_p, cap_p, _ = run(p, fx, st, steps)
    learned, its_l, cap_l, (acc, fb, _, judge) = run(p, fx, st, steps, w)
    print(f"NY {ny}: iterations plain {its_p} learned {its_l}; accepted {acc}, fell back {fb}, judge {judge:.2e}")
    assert cap_p == 0 and cap_l == 0
    assert its_l < its_p, (its_l, its_p)
    # the residual test accepts most guesses, and an accepted root is the plain solve's
    assert acc > 0.5 * (acc + fb), (acc, fb)
    assert judge < 1e-8, judge
    o = oracle_lib.Oracle(p, fx, st, None, double=True)
    for it in range(steps):
        o.step(it)
    NZ, NY = p["NZ"], p["NY"]
    s_ref = o.get("slip").reshape(NZ, NY)
    scale = np.abs(s_ref).max()
    err_p = np.abs(plain["slip"] - s_ref).max() / scale
    err_l = np.abs(learned["slip"] - s_ref).max() / scale
    # tolerance of the rate-and-state parity tests (FP32 path against the FP64 oracle)
    assert err_p < 2e-3 and err_l < 2e-3
    assert np.abs(learned["slip"] - plain["slip"]).max() / scale < 1e-4
    assert abs(err_l - err_p) < 1e-4
