"""The learned collision predictor: FP64 oracle (CPU) and CUDA kernels (B200).

Tolerances: the CUDA network stores inputs, weights, activations and
backpropagated dZ in BF16 and accumulates in FP32.  The oracle emulates the
BF16 storage, so gradients agree to FP32 summation-order error: per-tensor
relative L2 error <= 2e-2, loss relative error <= 1e-3, probabilities within
2e-3.  Adam is compared on the same gradient to 1e-6 absolute.
"""
import numpy as np
import pytest

import mlp_oracle as MO


def _rand_params(rng, n_params, scale=0.2):
    return (rng.standard_normal(n_params) * scale).astype(np.float64)


def _n_params():
    n = 0
    for l in range(MO.LAYERS + 1):
        nin = MO.IN_PAD if l == 0 else MO.HID
        nout = 1 if l == MO.LAYERS else MO.HID
        n += nout * nin + nout
    return n


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    params = _rand_params(rng, _n_params(), 0.1)
    X = MO.features(rng.uniform(-np.pi, np.pi, (6, 6)))
    y = (rng.random(6) < 0.5).astype(np.float64)
    loss, g, _ = MO.forward_backward(params, X, y, emulate_bf16=False)
    idx = rng.choice(len(params), 40, replace=False)
    # include a bias of every layer and the output layer
    idx = np.concatenate([idx, [len(params) - 1, len(params) - 2]])
    for i in idx:
        e = np.zeros_like(params)
        e[i] = 1e-6
        lp, _, _ = MO.forward_backward(params + e, X, y, emulate_bf16=False)
        lm, _, _ = MO.forward_backward(params - e, X, y, emulate_bf16=False)
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -2.5], np.float32)
    r = MO.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0            # exactly half an ulp: tie -> even
    assert r[2] == 1.0            # below the tie
    assert r[3] == 1.0 + 2 ** -7  # above the tie
    assert r[4] == -2.5


def _gpu_setup(n=512, seed=1):
    import torch
    from gpuprm_b200.mlp import CollisionMLP
    rng = np.random.default_rng(seed)
    q = rng.uniform(-np.pi, np.pi, (n, 6)).astype(np.float32)
    y = (rng.random(n) < 0.4).astype(np.float32)
    mlp = CollisionMLP(6, seed=seed)
    q_soa = torch.tensor(np.ascontiguousarray(q.T), device="cuda:0")
    y_t = torch.tensor(y, device="cuda:0")
    return mlp, q, y, q_soa, y_t


@pytest.mark.gpu
@pytest.mark.parametrize("path", ["tcgen05", "mma_sync"])
def test_gpu_gradients_match_oracle(path):
    mlp, q, y, q_soa, y_t = _gpu_setup()
    mlp.set_training(path)
    params = mlp.get_params().astype(np.float64)
    g_gpu, loss_gpu = mlp.gradients(q_soa, y_t)
    loss, g, _ = MO.forward_backward(params, MO.features(q), y.astype(np.float64), emulate_bf16=True)
    assert abs(loss_gpu - loss) <= 1e-3 * abs(loss)
    G, Gg = MO.unpack(g), MO.unpack(g_gpu.astype(np.float64))
    for k in G:
        num = np.linalg.norm(Gg[k] - G[k])
        den = np.linalg.norm(G[k]) + 1e-12
        assert num / den <= 2e-2, (k, num / den)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [37, 128, 4096, 5003])
def test_gpu_tensor_core_gradients_match_mma_sync(n):
    """The tcgen05 training GEMMs (TMA-loaded operands, split-K weight
    gradients reduced in a fixed order) and the mma.sync GEMMs compute the
    same gradients up to FP32 summation order and BF16 rounding of the
    activations; sizes cover a partial tile, one tile, the training batch
    and a batch that is not a multiple of the K step."""
    mlp, q, y, q_soa, y_t = _gpu_setup(n=n, seed=11)
    mlp.set_params(mlp.get_params() * 2.0)
    mlp.set_training("mma_sync")
    g_ref, l_ref = mlp.gradients(q_soa, y_t)
    g_ref2, _ = mlp.gradients(q_soa, y_t)
    mlp.set_training("tcgen05")
    g_tc, l_tc = mlp.gradients(q_soa, y_t)
    g_tc2, _ = mlp.gradients(q_soa, y_t)
    assert mlp.device_status() == 0
    # every reduction runs in a fixed order: the same bits on every run
    np.testing.assert_array_equal(g_tc, g_tc2)
    np.testing.assert_array_equal(g_ref, g_ref2)
    assert abs(l_tc - l_ref) <= 1e-3 * abs(l_ref)
    G, Gt = MO.unpack(g_ref.astype(np.float64)), MO.unpack(g_tc.astype(np.float64))
    for k in G:
        num = np.linalg.norm(Gt[k] - G[k])
        den = np.linalg.norm(G[k]) + 1e-12
        assert num / den <= 2e-2, (k, num / den)


@pytest.mark.gpu
@pytest.mark.parametrize("path", ["tcgen05", "mma_sync"])
def test_gpu_training_is_reproducible(path):
    """Two trainings from the same initial weights on the same labels and
    seed end with identical weights (no reduction depends on scheduling)."""
    import torch
    from gpuprm_b200.mlp import CollisionMLP
    rng = np.random.default_rng(8)
    n = 3 * 4096 + 100
    q = torch.tensor(rng.uniform(-np.pi, np.pi, (6, n)).astype(np.float32), device="cuda:0")
    y = torch.tensor((rng.random(n) < 0.4).astype(np.float32), device="cuda:0")
    params = []
    for _ in range(2):
        m = CollisionMLP(6, seed=3)
        m.set_training(path)
        m.train(q, y, epochs=2, batch=4096, lr=1e-3, seed=9)
        assert m.device_status() == 0
        params.append(m.get_params())
    np.testing.assert_array_equal(params[0], params[1])


@pytest.mark.gpu
def test_gpu_adam_matches_oracle():
    mlp, q, y, q_soa, y_t = _gpu_setup(seed=2)
    w0 = mlp.get_params().astype(np.float64)
    g, _ = mlp.gradients(q_soa, y_t)
    mlp.adam_step(1e-3)
    w1 = mlp.get_params().astype(np.float64)
    want, _, _ = MO.adam(w0, g.astype(np.float64), np.zeros_like(w0), np.zeros_like(w0), 1, lr=1e-3)
    assert np.max(np.abs(w1 - want)) <= 1e-6


@pytest.mark.gpu
def test_gpu_predict_matches_oracle():
    mlp, q, y, q_soa, y_t = _gpu_setup(n=3000, seed=3)
    p_gpu = mlp.predict(q_soa).cpu().numpy()
    _, _, p = MO.forward_backward(mlp.get_params().astype(np.float64), MO.features(q), y.astype(np.float64))
    assert np.max(np.abs(p_gpu - p)) <= 2e-3


@pytest.mark.gpu
@pytest.mark.parametrize("path", ["tcgen05", "mma_sync"])
def test_training_learns_exact_checker_labels(path):
    """A short training run on exact-checker labels of the hull6 scene
    lowers the loss and beats the constant predictor (both training paths)."""
    import torch
    from gpuprm_b200 import scenes
    from gpuprm_b200.configspace import RobotConfigspace
    from gpuprm_b200.mlp import CollisionMLP
    sc = scenes.make_hull6(0)
    cs = RobotConfigspace(sc, dq=0.01)
    cs.init()
    n = 1 << 16
    q = torch.tensor(np.ascontiguousarray(scenes.uniform_configs(sc, n, 7).T), device="cuda:0")
    codes = torch.zeros(n, dtype=torch.int32, device="cuda:0")
    cs.check_configs_device(q, codes)
    y = (codes != 0).float()
    mlp = CollisionMLP(6, seed=4)
    mlp.set_training(path)
    losses = mlp.train(q, y, epochs=4, batch=4096, lr=1e-3, seed=5)
    assert losses[-1] < losses[0]
    qt = torch.tensor(np.ascontiguousarray(scenes.uniform_configs(sc, 8192, 8).T), device="cuda:0")
    ct = torch.zeros(8192, dtype=torch.int32, device="cuda:0")
    cs.check_configs_device(qt, ct)
    p = mlp.predict(qt)
    torch.cuda.synchronize()
    acc = ((p > 0.5) == (ct != 0)).float().mean().item()
    base = max((ct != 0).float().mean().item(), 1 - (ct != 0).float().mean().item())
    assert acc > base + 0.05, (acc, base)


@pytest.mark.gpu
@pytest.mark.parametrize("path", ["tcgen05", "tcgen05_layers"])
@pytest.mark.parametrize("n,ndof", [(5000, 6), (131, 7), (1, 4)])
def test_gpu_tensor_core_inference_matches_training_path_and_oracle(n, ndof, path):
    """The tcgen05 inference paths compute the training forward's function
    (same BF16 roundings, FP32 accumulation in another order)."""
    import torch
    from gpuprm_b200.mlp import CollisionMLP
    rng = np.random.default_rng(7)
    q = rng.uniform(-np.pi, np.pi, (n, ndof)).astype(np.float32)
    mlp = CollisionMLP(ndof, seed=9)
    mlp.set_params(mlp.get_params() * 3.0)      # larger weights: outputs away from 0.5
    q_soa = torch.tensor(np.ascontiguousarray(q.T), device="cuda:0")
    mlp.set_inference("training")
    p_ref = mlp.predict(q_soa).cpu().numpy()
    mlp.set_inference(path)
    p_tc = mlp.predict(q_soa).cpu().numpy()
    assert mlp.device_status() == 0
    assert np.max(np.abs(p_tc - p_ref)) <= 2e-3
    _, _, p = MO.forward_backward(mlp.get_params().astype(np.float64), MO.features(q), np.zeros(n))
    # the tripled weights amplify a one-ulp BF16 difference of an activation
    # (FP32 summation order decides a rounding) up to the output: bound the
    # worst case loosely and the typical error tightly
    assert np.max(np.abs(p_tc - p)) <= 1e-2
    if n >= 100:
        assert np.median(np.abs(p_tc - p)) <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 127, 128, 129, 18944, 18944 + 128, 3 * 18944 + 5, 100003, 1 << 20])
def test_gpu_fused_inference_equals_layered_kernels(n):
    """The fused kernel (all layers of a tile on one SM, two tiles in
    flight per CTA) and the per-layer tcgen05 kernels issue the same MMAs
    in the same K order and split the output head the same way, so they
    give the same bits.  Sizes cover a partial tile, exact tiles, an odd
    number of tiles per CTA and several tile pairs per CTA (148 CTAs x 128
    rows = 18944 rows per wave)."""
    import torch
    from gpuprm_b200.mlp import CollisionMLP
    rng = np.random.default_rng(n)
    q = rng.uniform(-np.pi, np.pi, (n, 6)).astype(np.float32)
    mlp = CollisionMLP(6, seed=3)
    mlp.set_params(mlp.get_params() * 2.0)
    q_soa = torch.tensor(np.ascontiguousarray(q.T), device="cuda:0")
    mlp.set_inference("tcgen05_layers")
    p_l = mlp.predict(q_soa).cpu().numpy()
    mlp.set_inference("tcgen05")
    p_f = mlp.predict(q_soa).cpu().numpy()
    p_f2 = mlp.predict(q_soa).cpu().numpy()
    assert mlp.device_status() == 0
    assert np.array_equal(p_f, p_f2)
    assert np.all(np.isfinite(p_f))
    assert np.array_equal(p_f, p_l), np.max(np.abs(p_f - p_l))


def test_gelu_tanh_form_evaluation():
    """The device evaluates GELU(z) = z/2 (1 + tanh(k (z + c z^3))) as
    u = z (k + kc z^2), hz + hz tanh(u), hz = z/2, in FP32 with the
    constants rounded to FP32; with an exact tanh that order stays within
    1e-6 |z| of the oracle's FP64 function, and a tanh relative error of
    2^-11 (tanh.approx.f32) moves GELU by at most |z| 2^-12 - below half a
    BF16 ulp of the activation for |z| >= 0.1.  The derivative the device
    uses, (1 + t)/2 + hz (1 - t^2) k (1 + 3 c z^2), is the oracle's, pinned
    here by central differences."""
    z = np.linspace(-12.0, 12.0, 48001)
    f = np.float32
    z32 = z.astype(f)
    kc, k = f(0.035677408136300125), f(0.7978845608028654)
    u = z32 * (z32 * z32 * kc + k).astype(f)
    t = np.tanh(u.astype(np.float64)).astype(f)
    hz = z32 * f(0.5)
    g32 = (hz.astype(np.float64) * t + hz).astype(f)
    ref = MO.gelu(z32.astype(np.float64))
    assert np.max(np.abs(g32 - ref) / np.maximum(np.abs(z32), 1e-3)) <= 1e-6
    err = np.abs(0.5 * z * np.tanh(u) * 2.0 ** -11)
    assert np.all(err <= np.abs(z) * 2.0 ** -12 + 1e-30)
    h = 1e-6
    fd = (MO.gelu(z + h) - MO.gelu(z - h)) / (2 * h)
    assert np.max(np.abs(fd - MO.gelu_grad(z))) <= 1e-7
    # GELU's limits: z for large z, 0 for very negative z
    assert abs(MO.gelu(np.array([12.0]))[0] - 12.0) < 1e-12 and abs(MO.gelu(np.array([-12.0]))[0]) < 1e-12
