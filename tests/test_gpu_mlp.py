"""Learned plasticity surrogate on the GPU: gradients of the project's BF16
tensor-core backward pass against the CPU reference (oracle/mlp_ref.py),
training on pairs logged by the plain solver, and an A/B run of the solver
with and without the network (accuracy of F against the exact return map and
the particles it takes off the SVD path)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def synthetic_pairs(n, seed=0, t0=0.975, t1=1.0075):
    """Exact return-map pairs (numpy SVD + clamp) for random out-of-band trial F."""
    rng = np.random.default_rng(seed)
    out = []
    while sum(o.shape[0] for o in out) < n:
        U = np.linalg.qr(rng.standard_normal((n, 3, 3)))[0]
        V = np.linalg.qr(rng.standard_normal((n, 3, 3)))[0]
        U *= np.sign(np.linalg.det(U))[:, None, None]
        V *= np.sign(np.linalg.det(V))[:, None, None]
        s = rng.uniform(0.955, 1.02, (n, 3))
        Fh = U @ (s[:, :, None] * np.transpose(V, (0, 2, 1)))
        sc = np.clip(s, t0, t1)
        Fe = U @ (sc[:, :, None] * np.transpose(V, (0, 2, 1)))
        jp = rng.uniform(0.6, 1.0, n)
        p = np.concatenate([Fh.reshape(n, 9), jp[:, None], Fe.reshape(n, 9), (jp * np.prod(s / sc, 1))[:, None]], 1)
        out.append(p[(np.abs(s - sc) > 1e-4).any(1)])
    return np.concatenate(out)[:n].astype(np.float32)


@pytest.fixture(scope="module")
def mlp_mod(gpu_lib):
    from mpm_snow_sim2d_b200 import mlp
    return mlp


def test_gradient_matches_cpu_oracle(mlp_mod):
    from oracle import mlp_ref
    pairs = synthetic_pairs(512, seed=3)
    net = mlp_mod.Mlp(seed=11)
    norm = mlp_mod.normalization(pairs)
    net.set_normalization(*norm)
    g_gpu, l_gpu = net.gradient(pairs)
    l_ref, g_ref = mlp_ref.loss_and_grad(net.params(), pairs, norm, bf16_emulation=True)
    l_64, g_64 = mlp_ref.loss_and_grad(net.params(), pairs, norm, bf16_emulation=False)
    rel = np.linalg.norm(g_gpu - g_ref) / np.linalg.norm(g_ref)
    rel64 = np.linalg.norm(g_gpu - g_64) / np.linalg.norm(g_64)
    assert abs(l_gpu - l_ref) <= 1e-3 * l_ref
    assert rel < 1e-2, f"gradient vs BF16-emulated reference: {rel:.3e}"
    assert rel64 < 5e-2, f"gradient vs FP64 reference: {rel64:.3e}"
    for name in ("W1", "W2", "W3", "W4", "b4"):
        o, sz = mlp_mod.OFF[name]
        r = np.linalg.norm(g_gpu[o:o + sz] - g_ref[o:o + sz]) / max(np.linalg.norm(g_ref[o:o + sz]), 1e-30)
        assert r < 2e-2, f"{name}: {r:.3e}"


def test_training_on_logged_pairs(mlp_mod):
    from mpm_snow_sim2d_b200 import mlp_train
    pairs = mlp_train.collect_pairs(300_000, seed=5, W=48, steps=200, per_scene=100_000, verbose=False)
    assert pairs.shape[0] > 100_000
    net, info = mlp_train.train(pairs, steps=1500, batch=8192, lr=2e-3, seed=1)
    loss = info["loss"]
    assert loss[-50:].mean() < 0.05 * loss[:10].mean()
    # the network corrects F far better than leaving it unclamped
    assert info["heldout_rel_err_median"] < 0.2 * info["identity_rel_err_median"], info
    pytest.trained = net


def test_solver_with_learned_return_map(mlp_mod):
    from mpm_snow_sim2d_b200 import Solver, _lib
    from mpm_snow_sim2d_b200 import mlp_train
    net = getattr(pytest, "trained", None)
    if net is None:
        pytest.skip("needs the network trained above")
    sc = mlp_train.impact_scene(5.0, seed=424242, W=48, steps=120)
    with Solver.from_scene(sc) as plain:
        plain.Step(120)
        ref = plain.get_state()
    with Solver.from_scene(sc) as s:
        s.set_plasticity(_lib.PLASTIC_MLP, net, 1e-3)
        s.Step(120)
        got = s.get_state()
        acc, rej = s.mlp_stats()
        flags = s.status()
    assert flags & 1 == 0
    assert acc + rej > 1000
    rel_F = np.linalg.norm(got.elastic_f - ref.elastic_f) / np.linalg.norm(ref.elastic_f)
    g2p = lambda t: t.get("g2p", t.get("g2p2g", 0.0))  # the fused transfer reports its kernel as g2p2g
    rel_x = np.linalg.norm(got.position - ref.position) / np.linalg.norm(ref.position)
    print(f"learned return map: accepted {acc}, fell back {rej}, rel F {rel_F:.2e}, rel x {rel_x:.2e}")
    assert rel_F <= 1e-3
    assert rel_x <= 1e-4
    # every accepted prediction passed the residual check at 1e-3; a useful
    # network takes most out-of-band particles off the SVD
    assert acc > rej


def test_pretrained_weights_take_particles_off_the_svd(mlp_mod):
    """The shipped network (mpm_snow_sim2d_b200/data) on an impact it was not
    trained on: most out-of-band particles skip the SVD, and F stays within
    1e-3 of the exact return map's run."""
    from mpm_snow_sim2d_b200 import Solver, _lib
    from mpm_snow_sim2d_b200 import mlp_train
    net = mlp_mod.Mlp.load(mlp_mod.DEFAULT_WEIGHTS)
    sc = mlp_train.impact_scene(6.5, seed=777001, W=48, steps=300)
    with Solver.from_scene(sc) as plain:
        t_plain = plain.step_profiled(300)
        ref = plain.get_state()
    with Solver.from_scene(sc) as s:
        s.set_plasticity(_lib.PLASTIC_MLP, net, 1e-3)
        t_mlp = s.step_profiled(300)
        got = s.get_state()
        acc, rej = s.mlp_stats()
    rel_F = np.linalg.norm(got.elastic_f - ref.elastic_f) / np.linalg.norm(ref.elastic_f)
    g2p = lambda t: t.get("g2p", t.get("g2p2g", 0.0))  # the fused transfer reports its kernel as g2p2g
    print(f"pretrained: accepted {acc}, fell back {rej}, rel F {rel_F:.2e}, "
          f"return map {t_plain['return_map']:.2f} ms -> {t_mlp['return_map']:.2f} ms, "
          f"G2P {g2p(t_plain) + t_plain['return_map']:.2f} ms -> {g2p(t_mlp) + t_mlp['return_map']:.2f} ms "
          f"over 300 steps")
    assert acc > 4 * rej
    assert rel_F <= 1e-3
