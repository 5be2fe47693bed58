"""Generates tests/golden/*.npz: outputs of the reference's own correlation kernels.

TEST INFRASTRUCTURE.  Needs a CUDA GPU and ``oracle/_ref`` (built by
``oracle/build_ref.py`` from HI-SLAM2's ``src/correlation_kernels.cu`` and
``src/altcorr_kernel.cu``, unmodified).  Every input is drawn from a seeded
generator and stored next to the reference output, so ``test_golden.py`` can
check the CPU oracle against the reference without a GPU.

Usage: ``python tests/golden/make_golden.py [outdir]``.
"""

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import build_ref  # noqa: E402


def lookup_inputs(g, N, H1, W1, H2, W2, spread, integer=False):
    vol = torch.randn(N, H1, W1, H2, W2, generator=g)
    x = -spread + (W2 - 1 + 2 * spread) * torch.rand(N, H1, W1, generator=g)
    y = -spread + (H2 - 1 + 2 * spread) * torch.rand(N, H1, W1, generator=g)
    if integer:
        x, y = torch.round(x), torch.round(y)
    return vol, torch.stack([x, y], 1).contiguous()


def main(outdir=HERE):
    ref = build_ref.load()
    if ref is None:
        raise SystemExit("oracle/_ref is not built (python oracle/build_ref.py)")
    dev = torch.device("cuda:0")
    g = torch.Generator().manual_seed(1234)
    cases = {}
    for name, dtype, r, integer in (("corr_index_f32_r3", torch.float32, 3, False),
                                    ("corr_index_f32_r4_int", torch.float32, 4, True),
                                    ("corr_index_f16_r2", torch.float16, 2, False)):
        vol, crd = lookup_inputs(g, 2, 5, 6, 7, 8, 4.0, integer)
        vol = vol.to(dtype)
        out, = ref.corr_index_forward(vol.to(dev), crd.to(dev), r)
        gr = torch.randn(out.shape, generator=g).to(dtype)
        vg, = ref.corr_index_backward(vol.to(dev), crd.to(dev), gr.to(dev), r)
        cases[name] = dict(volume=vol.numpy(), coords=crd.numpy(), radius=np.int64(r), corr=out.cpu().numpy(),
                           corr_grad=gr.numpy(), volume_grad=vg.cpu().numpy())
    for name, r in (("altcorr_f32_r2", 2), ("altcorr_f32_r3", 3)):
        B, N, C, H, W, M = 1, 3, 16, 6, 7, 4
        f1 = torch.randn(B, N, C, H, W, generator=g)
        f2 = torch.randn(B, N, C, H, W, generator=g)
        ii = torch.randint(0, N, (M,), generator=g)
        jj = torch.randint(0, N, (M,), generator=g)
        crd = torch.stack([-2 + (W + 3) * torch.rand(B, M, H, W, generator=g),
                           -2 + (H + 3) * torch.rand(B, M, H, W, generator=g)], 2).contiguous()
        out, = ref.altcorr_forward(f1.to(dev), f2.to(dev), crd.to(dev), ii.to(dev), jj.to(dev), r)
        gr = torch.randn(out.shape, generator=g)
        g1, g2 = ref.altcorr_backward(f1.to(dev), f2.to(dev), crd.to(dev), ii.to(dev), jj.to(dev), gr.to(dev), r)
        cases[name] = dict(fmap1=f1.numpy(), fmap2=f2.numpy(), coords=crd.numpy(), ii=ii.numpy(), jj=jj.numpy(),
                           radius=np.int64(r), corr=out.contiguous().cpu().numpy(), grad=gr.numpy(),
                           fmap1_grad=g1.cpu().numpy(), fmap2_grad=g2.cpu().numpy())
    os.makedirs(outdir, exist_ok=True)
    for name, arrays in cases.items():
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **arrays)
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
