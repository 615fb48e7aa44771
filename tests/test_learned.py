"""The learned schedule: the NumPy reference (CPU), the CUDA inference /
gradient / training kernels against it (GPU), the device features, and
solves in learned mode (bit-identical answers, and what the trained network
gains over the reference heuristic it falls back to)."""
import os

import numpy as np
import pytest

import ecl_mst as E
import mlp_ref as R
import oracle_lib as O


def _rand_problem(seed, B=200):
    rng = np.random.default_rng(seed)
    p = E.mlp_init(seed, mean=rng.normal(0, 1, 16), std=rng.uniform(0.5, 2, 16))
    x = rng.normal(0, 1, (B, 16)).astype(np.float32)
    t = rng.normal(0, 1, (B, 2)).astype(np.float32)
    return p, x, t


def test_numpy_reference_gradient_matches_finite_differences():
    p, x, t = _rand_problem(1, B=16)
    p = p.astype(np.float64)
    loss, g = R.loss_and_grad(p, x, t)
    rng = np.random.default_rng(2)
    for i in rng.choice(E.MLP_TRAINABLE, 40, replace=False):
        h = 1e-6
        q1, q2 = p.copy(), p.copy()
        q1[i] += h
        q2[i] -= h
        fd = (R.loss_and_grad(q1, x, t)[0] - R.loss_and_grad(q2, x, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), i


def test_weights_file_has_the_blob_layout():
    if not os.path.exists(E.WEIGHTS_PATH):
        pytest.skip("no trained weights shipped")
    w = np.fromfile(E.WEIGHTS_PATH, np.float32)
    assert w.size == E.MLP_PARAMS and np.isfinite(w).all()
    assert (w[-16:] > 0).all()  # feature std


@pytest.mark.gpu
def test_cuda_forward_matches_numpy():
    p, x, _ = _rand_problem(3)
    y = E.mlp_forward(p, x)
    ref, _ = R.forward(p, R.standardise(p, x))
    np.testing.assert_allclose(y, ref, rtol=1e-4, atol=1e-4)


@pytest.mark.gpu
def test_cuda_gradient_matches_numpy():
    p, x, t = _rand_problem(4)
    xs = R.standardise(p, x).astype(np.float32)
    g, loss = E.mlp_grad(p, xs, t)
    ref_loss, ref_g = R.loss_and_grad(p, xs, t)
    assert abs(loss - ref_loss) <= 1e-4 * max(1, abs(ref_loss))
    np.testing.assert_allclose(g, ref_g, rtol=1e-3, atol=2e-5)


@pytest.mark.gpu
def test_cuda_training_fits_a_smooth_target():
    rng = np.random.default_rng(5)
    x = rng.normal(0, 1, (512, 16)).astype(np.float32)
    t = np.stack([np.tanh(x[:, 0] - x[:, 1]), 0.5 * x[:, 2] ** 2 - 0.3 * x[:, 3]], 1).astype(np.float32)
    p0 = E.mlp_init(6)
    l0 = R.loss_and_grad(p0, x, t)[0]
    p1, hist = E.mlp_train(p0, x, t, epochs=300, lr=3e-3)
    l1 = R.loss_and_grad(p1, x, t)[0]
    assert hist[-1] < 0.25 * hist[0] and l1 < 0.2 * l0


@pytest.mark.gpu
def test_device_features_match_host_statistics():
    import torch
    g = E.gen_rmat(16, 16, 0.57, 0.19, 0.19, 7, 1 << 24)
    dev = torch.device("cuda:0")
    ni, nl, ew = (torch.from_numpy(a).to(dev) for a in (g.nindex, g.nlist, g.eweight))
    f = E.graph_features(g.nodes, g.edges, ni.data_ptr(), nl.data_ptr(), ew.data_ptr())
    deg = np.diff(g.nindex)
    want = [np.log2(g.nodes), np.log2(g.edges), np.log2(deg.mean() + 1), np.log2(deg.max() + 1),
            deg.std() / deg.mean(), (deg == 0).mean(), (deg < 4).mean(), (deg >= 32).mean(),
            3 * g.nodes / g.edges]
    np.testing.assert_allclose(f[:9], want, rtol=1e-4, atol=1e-6)
    assert (np.diff(f[9:]) >= 0).all() and 0 <= f[9] and f[15] <= 1


@pytest.mark.gpu
@pytest.mark.parametrize("family", ["grid", "er", "rmat", "rgg"])
def test_solve_features_equal_the_feature_pass(family):
    """A learned solve takes its degree statistics from k_prep's vertex pass
    and sorts the weight sample beside it; the features it feeds the network
    are bit for bit those of the standalone feature pass (ecl_graph_features)
    that the training sweeps record."""
    import torch
    if not E.learned_load_default():
        pytest.skip("no trained weights shipped")
    dg = {"grid": lambda: E.gen_grid_device(700, 700, 3, 1 << 20),
          "er": lambda: E.gen_er_device(100_000, 16.0, 3, 1 << 24),
          "rmat": lambda: E.gen_rmat_device(17, 16, 0.57, 0.19, 0.19, 3, 1 << 30),
          "rgg": lambda: E.gen_rgg2d_device(400_000, 3.0, 3, 1 << 24)}[family]()
    assert dg.edges >= 1 << 20  # graphs below that keep the heuristic
    out = torch.empty(dg.edges, dtype=torch.uint8, device="cuda:0")
    want = E.graph_features(dg.nodes, dg.edges, dg.d_nindex, dg.d_nlist, dg.d_eweight)
    with E.Context(dg.nodes, dg.edges) as ctx:
        with pytest.raises(E.EclError):
            ctx.learned_features()  # no learned solve yet
        st = ctx.run_device(dg.nodes, dg.edges, dg.d_nindex, dg.d_nlist, dg.d_eweight, out.data_ptr(),
                            opts=E.make_opts(mode=E.THRESH_LEARNED), stats=True)
        assert st["status"] == 0
        got = ctx.learned_features()
    dg.close()
    np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
def test_learned_mode_keeps_the_answer(golden):
    rng = np.random.default_rng(8)
    p = E.mlp_init(9, mean=np.zeros(16), std=np.ones(16))
    p[-34 - 128:-34] = 0.0  # W3 = 0 ...
    p[-34:-32] = [-3.0, 3.0]  # ... and b3: quantile 2^-3, split 8 for any input
    E.learned_set_weights(p)
    ctx = E.Context(1 << 20, 1 << 24)
    for name, c in golden.items():
        got, st = ctx.run_host(E.Graph(c["nindex"], c["nlist"], c["eweight"]), E.make_opts(mode=E.THRESH_LEARNED))
        assert np.array_equal(got, c["inMST"]), name
    g = E.gen_rmat(16, 16, 0.57, 0.19, 0.19, 2, 1 << 24)
    want, _, _ = O.oracle_mst(g.nindex, g.nlist, g.eweight, *E.heuristic_threshold(g))
    got, st = ctx.run_host(g, E.make_opts(mode=E.THRESH_LEARNED))
    assert np.array_equal(got, want)
    ctx.close()
    if os.path.exists(E.WEIGHTS_PATH):
        E.learned_load_default()


@pytest.mark.gpu
def test_trained_network_gains_over_the_heuristic():
    """Held-out graphs (seeds the training never drew, train_filter.py's
    held-out range) of 200k-4M vertices from the four families: the learned
    schedule solves them faster than the reference heuristic in total, with
    the same answers. Each graph is timed best of three, the two schedules
    interleaved."""
    if not E.learned_load_default():
        pytest.skip("no trained weights shipped")
    import torch
    import train_filter as TF
    t_h = t_l = 0.0
    with E.Context(1 << 23, 300_000_000) as ctx:
        for i in range(12):
            dg, fam = TF.make_graph(TF.HELDOUT_SEED0 + i, 200_000, 4_000_000)
            out = torch.empty(max(dg.edges, 1), dtype=torch.uint8, device="cuda:0")
            best, answer = {}, {}
            for _ in range(2):
                for mode in (E.THRESH_HEURISTIC, E.THRESH_LEARNED):
                    best[mode] = min(best.get(mode, 1e30), TF.solve_ms(ctx, dg, out, E.make_opts(mode=mode), 1))
                    answer[mode] = out[: dg.edges].cpu().numpy().copy()
            assert np.array_equal(answer[E.THRESH_HEURISTIC], answer[E.THRESH_LEARNED]), (i, fam)
            t_h += best[E.THRESH_HEURISTIC]
            t_l += best[E.THRESH_LEARNED]
            dg.close()
    print(f"held-out: heuristic {t_h:.3f} ms, learned {t_l:.3f} ms, gain {t_h / t_l:.3f}x")
    assert t_h / t_l > 1.0
