"""The learned denoiser on the GPU, through the C ABI.

* the tensor-core 3x3 convolution (tcgen05 + TMEM + TMA) against a plain PyTorch
  fp32 convolution of the same bf16-rounded operands, for every channel count
  the U-Net uses (tolerance 2e-3 of the output scale: f32 accumulation order);
* its weight gradient against torch's, same tolerance;
* the whole network's loss and parameter gradients against the CPU oracle
  (oracle/unet_ref.py), which rounds to bf16 where the device stores bf16
  (tolerance: relative L2 error per layer < 5e-2, loss within 1e-3 relative);
* training lowers the loss, and inference pads arbitrary image sizes.
"""
import numpy as np
import pytest
import torch
import torch.nn.functional as F

pytestmark = pytest.mark.gpu


def _bf(a):
    return torch.tensor(a).to(torch.bfloat16).to(torch.float32)


def _ref_conv(x, w, bias=None, relu=False):
    xt = _bf(x).permute(0, 3, 1, 2)
    wt = _bf(w).permute(0, 3, 1, 2)
    y = F.conv2d(xt, wt, padding=1)
    if bias is not None:
        y = y + torch.tensor(bias).view(1, -1, 1, 1)
    if relu:
        y = F.relu(y)
    return y.permute(0, 2, 3, 1).numpy()


@pytest.mark.parametrize("cin,cout", [(16, 32), (32, 32), (32, 64), (64, 128), (96, 32), (128, 256), (192, 64),
                                      (384, 128), (256, 256), (32, 3), (16, 16)])
def test_conv_forward_matches_torch(gpu, cin, cout):
    rng = np.random.default_rng(cin * 1000 + cout)
    B, H, W = 2, 16, 32
    x = rng.standard_normal((B, H, W, cin)).astype(np.float32)
    w = (rng.standard_normal((cout, 3, 3, cin)) / np.sqrt(9 * cin)).astype(np.float32)
    b = rng.standard_normal(cout).astype(np.float32)
    y = gpu.conv3x3(x, w, bias=b, relu=False, f32_out=True)
    ref = _ref_conv(x, w, b)
    scale = np.abs(ref).max()
    assert np.abs(y - ref).max() <= 2e-3 * scale, (np.abs(y - ref).max(), scale)


@pytest.mark.parametrize("cin,cout,h,w", [(32, 32, 32, 80), (96, 32, 16, 16), (16, 48, 16, 48), (64, 16, 48, 16)])
def test_conv_forward_tile_edges(gpu, cin, cout, h, w):
    """Small-Cout layers at other image sizes: a single 16-pixel column, tall and wide
    images, and 16 / 32 / 48 output channels."""
    rng = np.random.default_rng(cin + cout + h + w)
    x = rng.standard_normal((1, h, w, cin)).astype(np.float32)
    wt = (rng.standard_normal((cout, 3, 3, cin)) / np.sqrt(9 * cin)).astype(np.float32)
    b = rng.standard_normal(cout).astype(np.float32)
    y = gpu.conv3x3(x, wt, bias=b, relu=True, f32_out=True)
    ref = _ref_conv(x, wt, b, relu=True)
    scale = np.abs(ref).max()
    assert np.abs(y - ref).max() <= 2e-3 * scale, (np.abs(y - ref).max(), scale)


def test_conv_forward_relu_bf16_out(gpu):
    rng = np.random.default_rng(7)
    x = rng.standard_normal((1, 24, 48, 64)).astype(np.float32)
    w = (rng.standard_normal((64, 3, 3, 64)) / 24).astype(np.float32)
    y = gpu.conv3x3(x, w, relu=True, f32_out=False)
    ref = _ref_conv(x, w, relu=True)
    ref_bf = _bf(ref).numpy()
    # the device rounds the f32 accumulator to bf16 once: at most one bf16 ulp apart
    assert np.all(np.abs(y - ref_bf) <= np.abs(ref_bf) * 2 ** -7 + 1e-6)


@pytest.mark.parametrize("cin,cout", [(16, 32), (32, 64), (96, 32), (64, 128), (128, 256), (384, 128), (32, 16),
                                      (256, 256)])
def test_conv_wgrad_matches_torch(gpu, cin, cout):
    rng = np.random.default_rng(cin + 17 * cout)
    B, H, W = 2, 16, 32
    x = rng.standard_normal((B, H, W, cin)).astype(np.float32)
    g = rng.standard_normal((B, H, W, cout)).astype(np.float32)
    dw = gpu.conv3x3_wgrad(g, x)
    ref = torch.nn.grad.conv2d_weight(_bf(x).permute(0, 3, 1, 2), (cout, cin, 3, 3), _bf(g).permute(0, 3, 1, 2),
                                      padding=1).permute(0, 2, 3, 1).numpy()
    scale = np.abs(ref).max()
    assert np.abs(dw - ref).max() <= 2e-3 * scale, (np.abs(dw - ref).max(), scale)


def test_conv_rejects_bad_shapes(gpu):
    x = np.zeros((1, 8, 16, 24), np.float32)  # Cin not a multiple of 16
    w = np.zeros((16, 3, 3, 24), np.float32)
    with pytest.raises(gpu.WrkError):
        gpu.conv3x3(x, w)


def _images(rng, B, H, W):
    rgb = rng.gamma(0.6, 0.5, (B, H, W, 3)).astype(np.float32)
    alb = rng.uniform(0, 1, (B, H, W, 3)).astype(np.float32)
    nrm = rng.uniform(-1, 1, (B, H, W, 3)).astype(np.float32)
    tgt = (rgb * rng.uniform(0.5, 1.5, (B, H, W, 3))).astype(np.float32)
    return rgb, alb, nrm, tgt


def test_denoiser_gradients_match_oracle(gpu):
    import unet_ref

    rng = np.random.default_rng(3)
    B, H, W = 2, 64, 128
    rgb, alb, nrm, tgt = _images(rng, B, H, W)
    dn = gpu.Denoiser(seed=5)
    p = dn.get_params()
    # non-zero head so every layer's gradient is exercised
    p[-(3 * 9 * 32 + 3):] = (rng.standard_normal(3 * 9 * 32 + 3) * 0.05).astype(np.float32)
    dn.set_params(p)
    arrs = [gpu.DeviceArray.from_numpy(a) for a in (rgb, alb, nrm, tgt)]
    loss, g = dn.gradients(*arrs, B, H, W)
    rloss, rg = unet_ref.loss_and_grads(p, rgb, alb, nrm, tgt)
    assert abs(loss - rloss) <= 1e-3 * abs(rloss)
    o = 0
    for i, (cin, cout) in enumerate(unet_ref.LAYERS):
        n = cout * 9 * cin
        for name, sl in (("W", slice(o, o + n)), ("b", slice(o + n, o + n + cout))):
            a, r = g[sl], rg[sl]
            rel = np.linalg.norm(a - r) / max(np.linalg.norm(r), 1e-12)
            assert rel < 5e-2, f"layer {i} {name}: relative L2 error {rel:.3e}"
        o += n + cout


def test_denoiser_forward_matches_oracle(gpu):
    import unet_ref

    rng = np.random.default_rng(4)
    B, H, W = 1, 64, 128
    rgb, alb, nrm, _ = _images(rng, B, H, W)
    dn = gpu.Denoiser(seed=9)
    p = dn.get_params()
    p[-(3 * 9 * 32 + 3):] = (rng.standard_normal(3 * 9 * 32 + 3) * 0.05).astype(np.float32)
    dn.set_params(p)
    out = dn.infer(rgb, alb, nrm)
    ref = unet_ref.denoise(p, rgb, alb, nrm)
    err = np.abs(np.log1p(out) - np.log1p(ref)).max()
    assert err < 2e-2, err


def test_denoiser_training_lowers_loss_and_pads(gpu):
    rng = np.random.default_rng(6)
    B, H, W = 4, 64, 128
    rgb, alb, nrm, tgt = _images(rng, B, H, W)
    dn = gpu.Denoiser(seed=1)
    arrs = [gpu.DeviceArray.from_numpy(a) for a in (rgb, alb, nrm, tgt)]
    l0 = dn.train_step(*arrs, B, H, W, 1e-3)
    for _ in range(40):
        l1 = dn.train_step(*arrs, B, H, W, 1e-3)
    assert np.isfinite(l1) and l1 < 0.8 * l0, (l0, l1)
    # arbitrary sizes are padded internally; output keeps the input's shape
    small = dn.infer(rgb[0, :37, :53], alb[0, :37, :53], nrm[0, :37, :53])
    assert small.shape == (37, 53, 3) and np.isfinite(small).all() and (small >= 0).all()


def test_trained_denoiser_gains_on_held_out_scene(gpu):
    """The committed weights (trained by offlinerenderer_b200.denoise_train on scene
    seeds 101-108) on the held-out benchmark scene (scale test, seed 1): the
    denoised 4-spp image is far closer to an FP64-accumulated 1024-spp reference
    than the 4-spp render it came from, and closer than the plain 64-spp render."""
    import torch

    from offlinerenderer_b200 import denoise_train, quality, scenes

    sd = scenes.scale_test(256, 256, 4, seed=1)
    scene = gpu.Scene.from_data(sd)
    renderer = gpu.Renderer()
    st, cam = sd.settings, sd.camera
    ref = quality.reference(renderer, scene, cam, st, total_spp=1024, chunk=256)
    dn = gpu.Denoiser()
    denoise_train.load_weights(dn, denoise_train.DEFAULT_WEIGHTS)
    rgb, alb, nrm, _ = quality.render(renderer, scene, cam, st, 4, 0, torch)
    out = torch.empty_like(rgb)
    dn.infer_device(quality._Ptr(rgb), quality._Ptr(alb), quality._Ptr(nrm), 1, 256, 256, quality._Ptr(out))
    plain64, _, _, _ = quality.render(renderer, scene, cam, st, 64, 4, torch, guides=False)
    noisy, den, p64 = quality.relmse(rgb, ref), quality.relmse(out, ref), quality.relmse(plain64, ref)
    assert den < 0.1 * noisy and den < p64, (noisy, den, p64)
