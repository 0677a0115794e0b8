"""The learned denoiser's tensor-core kernels against FP32/FP64 references on the CPU."""
from __future__ import annotations

import numpy as np
import pytest

from webgpuraytracer_b200 import _lib

pytestmark = pytest.mark.gpu


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 bit patterns, round to nearest even."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) >> 16).astype(np.uint16)


def bf16_value(b: np.ndarray) -> np.ndarray:
    return (b.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("m,n,k", [(128, 32, 64), (300, 96, 200), (257, 16, 8), (1000, 256, 576), (64, 200, 1232)])
def test_tc_gemm_matches_fp32(m, n, k):
    rng = np.random.default_rng(m * 7 + n + k)
    a = bf16_bits(rng.standard_normal((m, k)).astype(np.float32))
    b = bf16_bits(rng.standard_normal((n, k)).astype(np.float32))
    c = np.zeros((m, n), np.float32)
    L = _lib.lib()
    rc = L.wgpt_gemm_bf16(0, _lib.ptr(a), _lib.ptr(b), _lib.ptr(c), m, n, k)
    assert rc == 0, _lib.STATUS_NAMES.get(rc, rc)
    ref = bf16_value(a).astype(np.float64) @ bf16_value(b).astype(np.float64).T
    err = np.abs(c - ref)
    # FP32 accumulation of k products of BF16 values (exact in FP32): rounding only
    tol = 1e-5 * np.sqrt(k) * np.abs(bf16_value(a)).max() * np.abs(bf16_value(b)).max() * 4
    assert err.max() <= max(tol, 1e-4), f"max abs error {err.max()} (tol {tol})"


# ------------------------------------------------------------------------ the learned denoiser
import oracle.kpcn_ref as kref
from webgpuraytracer_b200 import kpcn
from webgpuraytracer_b200 import renderer as rd
from webgpuraytracer_b200 import synth


def _random_image(h, w, seed):
    rng = np.random.default_rng(seed)
    noisy = (np.abs(rng.standard_normal((h, w, 4))) * 0.6).astype(np.float32)
    gbuf = rng.standard_normal((h, w, 12)).astype(np.float32)
    gbuf[..., 4:7] = rng.random((h, w, 3))
    gbuf[..., 11] = rng.random((h, w)) * 8.0
    target = (np.abs(rng.standard_normal((h, w, 4))) * 0.5).astype(np.float32)
    return noisy, gbuf, target


def test_kpcn_layout_and_params_roundtrip():
    k = kpcn.Kpcn(0, seed=3)
    assert k.n_params == kpcn.N_PARAMS == 729_168
    p = k.get_params()
    sl = kpcn.param_slices()
    w0 = p[sl["E0a"][0]].reshape(32, 9, 16)
    assert np.all(w0[:, :, 10:] == 0.0), "padded input channels start at zero"
    wo = p[sl["OUT"][0]].reshape(80, 32)
    assert np.all(wo[75:] == 0.0), "padded logits start at zero"
    q = p * 0.5
    k.set_params(q)
    np.testing.assert_array_equal(k.get_params(), q)
    k.close()


@pytest.mark.parametrize("h,w", [(40, 48), (33, 70)])
def test_kpcn_loss_and_gradients_match_fp64_reference(h, w):
    """Forward (filtered colour, loss) and backward (every parameter gradient) of the BF16
    tensor-core network against the float64 restatement with the same BF16-rounded inputs and
    weights.  Odd sizes exercise the partial pooling windows and the cropped upsampling."""
    noisy, gbuf, target = _random_image(h, w, h * 1000 + w)
    k = kpcn.Kpcn(0, seed=5)
    p = k.get_params()
    # larger output weights than the initialisation, so every layer carries gradient
    sl = kpcn.param_slices()
    p[sl["OUT"][0]] *= 10.0
    k.set_params(p)
    loss_g, grad_g, out_g = k.loss_and_grads(noisy, gbuf, target)
    loss_r, grad_r, out_r = kref.loss_and_grads(p, noisy, gbuf, target)
    assert abs(loss_g - loss_r) <= 0.02 * abs(loss_r), (loss_g, loss_r)
    np.testing.assert_allclose(out_g[..., :3], out_r, rtol=0.03, atol=0.02 * float(np.abs(out_r).max()))
    # BF16 activations and gradients (8-bit mantissa; ReLU masks of near-zero activations can
    # differ) bound the agreement: direction within cos > 0.99, magnitude within 20 %
    report = []
    for l in kpcn.LAYERS:
        for part, s in zip(("W", "b"), sl[l.name]):
            g, r = grad_g[s].astype(np.float64), grad_r[s]
            nr = np.linalg.norm(r)
            assert nr > 0, f"{l.name}.{part}: no gradient in the reference"
            cos = float(g @ r / (np.linalg.norm(g) * nr + 1e-30))
            rel = float(np.linalg.norm(g - r) / nr)
            report.append(f"{l.name}.{part} cos {cos:.4f} rel {rel:.3f}")
            assert cos > 0.99 and rel < 0.2, f"{l.name}.{part}: cosine {cos:.4f}, relative error {rel:.4f}"
    print("; ".join(report))
    k.close()


@pytest.mark.parametrize("h,w", [(40, 48), (33, 70)])
def test_kpcn_gradients_match_bf16_rounding_reference(h, w):
    """The same check against the restatement that rounds to bfloat16 where the kernels store
    bfloat16 (post-ReLU activations, pooled tensors, the gradients flowing into them, logit
    gradients): what remains is the kernels' FP32 accumulation order and the rounding points the
    restatement places slightly differently (sums of two gradient contributions, upsampled
    gradients), so the bound is a few percent (8 % per tensor, cosine 0.997) instead of twenty."""
    noisy, gbuf, target = _random_image(h, w, h * 1000 + w)
    k = kpcn.Kpcn(0, seed=5)
    p = k.get_params()
    sl = kpcn.param_slices()
    p[sl["OUT"][0]] *= 10.0
    k.set_params(p)
    loss_g, grad_g, out_g = k.loss_and_grads(noisy, gbuf, target)
    loss_r, grad_r, out_r = kref.loss_and_grads(p, noisy, gbuf, target, bf16_activations=True)
    assert abs(loss_g - loss_r) <= 2e-3 * abs(loss_r), (loss_g, loss_r)
    np.testing.assert_allclose(out_g[..., :3], out_r, rtol=5e-3, atol=2e-3 * float(np.abs(out_r).max()))
    report, worst = [], 0.0
    for l in kpcn.LAYERS:
        for part, s_ in zip(("W", "b"), sl[l.name]):
            g, r = grad_g[s_].astype(np.float64), grad_r[s_]
            nr = np.linalg.norm(r)
            cos = float(g @ r / (np.linalg.norm(g) * nr + 1e-30))
            rel = float(np.linalg.norm(g - r) / nr)
            worst = max(worst, rel)
            report.append(f"{l.name}.{part} cos {cos:.5f} rel {rel:.4f}")
            assert cos > 0.997 and rel < 0.08, f"{l.name}.{part}: cosine {cos:.5f}, relative error {rel:.4f}"
    print(f"worst {worst:.4f}: " + "; ".join(report))
    k.close()


def _example(seed, size, spp, target_spp):
    s = synth.small_scene(seed, size, size, 4)
    return kpcn.render_example(s, size, spp, target_spp, seed=seed, target_seed=10_000 + seed)


def test_kpcn_training_gains_over_atrous():
    """Trained on path-traced pairs of one scene family, the network denoises a held-out scene
    at 4 spp with lower display-space RMSE than the a-trous filter and than no filter."""
    size, spp, tspp = 128, 4, 512
    k = kpcn.Kpcn(0, seed=11)
    for seed in range(2, 26):
        k.add_example(*_example(seed, size, spp, tspp))
    losses = k.train(600, batch=8, crop=64, lr=1e-3, seed=3)
    assert np.all(np.isfinite(losses))
    assert losses[-50:].mean() < 0.6 * losses[:50].mean(), (losses[:50].mean(), losses[-50:].mean())
    noisy, gbuf, target = _example(1, size, spp, tspp)
    s = synth.small_scene(1, size, size, 4)
    r = rd.Renderer(size, size)
    r.set_scene(s, isgbuf=True)
    r.write_accum(noisy)
    r.write_gbuffer(gbuf)
    lin = k.denoise(r, exposure=1.0)
    dn = rd.Denoiser(r, passes=4)
    dn.execute()
    _, comp, _ = dn.read()
    ref = kpcn.tonemap(target)
    e_noisy = kpcn.rmse(noisy, target)
    e_kpcn = kpcn.rmse(lin, target)
    e_atrous = float(np.sqrt(np.mean((np.clip(comp[..., :3], 0, 1) - ref) ** 2)))
    print(f"display RMSE: noisy {e_noisy:.4f}  a-trous {e_atrous:.4f}  kpcn {e_kpcn:.4f}")
    assert e_kpcn < e_noisy
    assert e_kpcn < e_atrous
    r.close()
    k.close()


# ------------------------------------------------------------------------ data-parallel training
def test_kpcn_grads_match_whole_image_gradient():
    """wgpt_kpcn_grads over one crop covering the only example equals the whole-image gradient
    (up to the order of the floating-point atomics that sum the weight gradients)."""
    import torch
    noisy, gbuf, target = _random_image(64, 64, 11)
    k = kpcn.Kpcn(0, seed=5)
    k.add_example(noisy, gbuf, target)
    loss_ref, g_ref, _ = k.loss_and_grads(noisy, gbuf, target)
    g = torch.empty(k.n_params, dtype=torch.float32, device="cuda:0")
    loss = k.grads(1, 64, 123, g)
    assert abs(loss - loss_ref) <= 1e-5 * abs(loss_ref)
    gd = g.cpu().numpy().astype(np.float64)
    # split-K weight gradients are summed with float atomics over BF16 activations: the
    # run-to-run spread is ~1e-3 of the norm
    assert np.linalg.norm(gd - g_ref) <= 5e-3 * np.linalg.norm(g_ref)
    with pytest.raises(_lib.WgptError):
        k.grads(1, 64, 1, torch.empty(k.n_params, dtype=torch.float32))     # host memory is refused
    k.close()


def _learnable_image(h, w, seed):
    """A random noisy image, G-buffer, and as target a fixed function of the noisy image."""
    noisy, gbuf, _ = _random_image(h, w, seed)
    return noisy, gbuf, (noisy * 0.5).astype(np.float32)


def _blurred_image(h, w, seed):
    """A random noisy image, G-buffer, and as target its 3x3 box blur (clamped edges): a convex
    combination of input pixels, which the softmax-normalised kernels can represent."""
    noisy, gbuf, _ = _random_image(h, w, seed)
    p = np.pad(noisy, ((1, 1), (1, 1), (0, 0)), mode="edge")
    tgt = sum(p[dy:dy + h, dx:dx + w] for dy in range(3) for dx in range(3)) / 9.0
    return noisy, gbuf, tgt.astype(np.float32)


def test_kpcn_emulated_two_rank_steps_keep_weights_identical():
    """Two denoisers with different examples, one gradient sum per step (what all_reduce
    gives every rank), the mean applied on both: the weights stay bit-identical, the loss falls."""
    import torch
    ks = [kpcn.Kpcn(0, seed=2) for _ in range(2)]
    for r, k in enumerate(ks):
        for e in range(3):
            k.add_example(*_blurred_image(64, 64, 100 * r + e))
    gs = [torch.empty(ks[0].n_params, dtype=torch.float32, device="cuda:0") for _ in ks]
    first = last = None
    seq = []
    for step in range(12):
        # each rank keeps its batch (seed r), so the summed loss is of the same data every step
        losses = [k.grads(2, 32, r, g) for r, (k, g) in enumerate(zip(ks, gs))]
        total = gs[0] + gs[1]
        torch.cuda.synchronize()
        for k in ks:
            k.apply(total, 0.5, 2e-4)   # small steps: a fixed 2 x 32^2 batch overshoots at 1e-3
        seq.append(sum(losses))
        first = first if first is not None else sum(losses)
        last = sum(losses)
    print("summed losses:", " ".join(f"{v:.4f}" for v in seq))
    assert np.array_equal(ks[0].get_params(), ks[1].get_params())
    assert last < first
    for k in ks:
        k.close()


def test_kpcn_train_data_parallel_single_rank():
    k = kpcn.Kpcn(0, seed=4)
    for e in range(2):
        k.add_example(*_learnable_image(64, 64, 300 + e))
    losses = kpcn.train_data_parallel(k, 30, batch=4, crop=64, lr=2e-3, seed=1)
    assert np.isfinite(losses).all() and losses[-5:].mean() < losses[:5].mean()
    k.close()


@pytest.mark.parametrize("h,w", [(40, 48), (33, 70), (96, 160)])
def test_kpcn_pipelined_convolutions_equal_per_tile(h, w):
    """The warp-specialised TMA convolution (default) against the one-CTA-per-tile kernel: the
    same MMAs accumulate in the same order into tensor memory, so the filtered output is identical
    bit for bit.  The loss, the filter stages' input gradients and the weight gradients are sums
    taken with FP32 atomics, whose order differs from run to run in either mode; a last-bit
    difference can flip the BF16 rounding of a data gradient further down, so the gradients are
    compared by norm, at the bound the whole-image gradient check uses for run-to-run spread."""
    noisy, gbuf, target = _random_image(h, w, h * 7 + w)
    k = kpcn.Kpcn(0, seed=9)
    p = k.get_params()
    sl = kpcn.param_slices()
    p[sl["OUT"][0]] *= 10.0
    k.set_params(p)
    L = _lib.lib()
    res = []
    for mode in (0, 1):
        assert L.wgpt_kpcn_set_conv_mode(k.h, mode) == 0
        res.append(k.loss_and_grads(noisy, gbuf, target))
    (l0, g0, o0), (l1, g1, o1) = res
    np.testing.assert_array_equal(o0, o1)
    assert abs(l0 - l1) <= 1e-6 * abs(l0)
    g0, g1 = g0.astype(np.float64), g1.astype(np.float64)
    assert np.linalg.norm(g1 - g0) <= 5e-3 * np.linalg.norm(g0)
    assert float(g0 @ g1) / (np.linalg.norm(g0) * np.linalg.norm(g1)) > 0.99999
    k.close()


def test_kpcn_pipelined_denoise_equals_per_tile():
    """1080p inference through both convolution kernels gives the same image bit for bit."""
    size_w, size_h = 1920, 1080
    s = synth.small_scene(1, size_w, size_h, 4)
    s.camera.aspect = size_w / size_h
    r = rd.Renderer(size_w, size_h)
    r.set_scene(s, isgbuf=True)
    r.render_gbuffer()
    r.reset()
    r.render(tsize=size_w, reps=2)
    k = kpcn.Kpcn(0, seed=4)
    L = _lib.lib()
    outs = []
    for mode in (0, 1):
        assert L.wgpt_kpcn_set_conv_mode(k.h, mode) == 0
        lin = k.denoise(r)
        outs.append((lin, r.read_output()))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
    k.close()
    r.close()


@pytest.mark.parametrize("h,w", [(40, 48), (67, 130)])
def test_kpcn_inference_tail_equals_training_forward(h, w):
    """Inference runs the output layer, the softmaxes and the first filter stage fused in one
    kernel and the last two stages from stored kernels; training runs the output layer as a GEMM
    into FP32 logits and the filter stages from those.  The arithmetic of every value is the
    same, so the filtered image is identical bit for bit."""
    noisy, gbuf, target = _random_image(h, w, h * 31 + w)
    k = kpcn.Kpcn(0, seed=6)
    p = k.get_params()
    sl = kpcn.param_slices()
    p[sl["OUT"][0]] *= 10.0          # sharper kernels than the initialisation's
    k.set_params(p)
    _, _, out_train = k.loss_and_grads(noisy, gbuf, target)
    s = synth.small_scene(1, w, h, 4)
    r = rd.Renderer(w, h)
    r.set_scene(s, isgbuf=True)
    r.write_accum(noisy)
    r.write_gbuffer(gbuf)
    out_infer = k.denoise(r, exposure=1.0)
    np.testing.assert_array_equal(out_infer[..., :3], out_train[..., :3])
    r.close()
    k.close()
