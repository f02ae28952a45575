"""Denoiser throughput: one inference and one training step, device-timed.

    python -m offlinerenderer_b200.denoise_bench [--size 1024 | --width W --height H] [--batch 1]
                                                 [--train-batch 8] [--repeat 1]

Loads the committed weights, denoises a batch of random images of size x size (or
width x height; inputs in device memory) and runs a training step on train-batch crops of
128x128; prints the device times (CUDA events on the denoiser's stream) and the
convolution throughput in TFLOP/s.
"""
from __future__ import annotations

import argparse
import json

from . import denoise_train, wrk

# 3x3 convolutions of the U-Net: (Cin, Cout padded to 16, level); FLOPs per
# full-resolution pixel = sum 2 * 9 * Cin * Cout / 4^level.
UNET_LAYERS = [(16, 32, 0), (32, 32, 0), (32, 64, 1), (64, 64, 1), (64, 128, 2), (128, 128, 2), (128, 256, 3),
               (256, 256, 3), (384, 128, 2), (128, 128, 2), (192, 64, 1), (64, 64, 1), (96, 32, 0), (32, 32, 0),
               (32, 16, 0)]
FLOP_PER_PX = sum(2 * 9 * ci * co / 4 ** lv for ci, co, lv in UNET_LAYERS)


_Ptr = wrk.TensorPtr


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=1024)
    ap.add_argument("--width", type=int, default=0, help="image width (default: --size)")
    ap.add_argument("--height", type=int, default=0, help="image height (default: --size)")
    ap.add_argument("--batch", type=int, default=1)
    ap.add_argument("--train-batch", type=int, default=8)
    ap.add_argument("--repeat", type=int, default=1)
    args = ap.parse_args()
    import torch

    dn = wrk.Denoiser()
    denoise_train.load_weights(dn)
    B = args.batch
    W, H = args.width or args.size, args.height or args.size
    x = torch.rand((B, H, W, 3), device="cuda")
    o = torch.empty_like(x)
    inf = []
    for _ in range(args.repeat):
        dn.infer_device(_Ptr(x), _Ptr(x), _Ptr(x), B, H, W, _Ptr(o))
        inf.append(dn.last_ms())
    tb = args.train_batch
    xb = torch.rand((tb, 128, 128, 3), device="cuda")
    tr = []
    for _ in range(args.repeat):
        dn.train_step(_Ptr(xb), _Ptr(xb), _Ptr(xb), _Ptr(xb), tb, 128, 128, 1e-5)
        tr.append(dn.last_ms())
    hp, wp = (H + 63) // 64 * 64, (W + 127) // 128 * 128
    out = {"infer_ms": min(inf), "infer_tflops": FLOP_PER_PX * B * hp * wp / (min(inf) / 1e3) / 1e12,
           "train_ms": min(tr), "train_tflops": 3 * FLOP_PER_PX * tb * 128 * 128 / (min(tr) / 1e3) / 1e12}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
