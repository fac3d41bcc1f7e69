"""Differentiable path: the adjoint kernel behind DFTTestFunction.

Checked against (a) torch autograd through the float64 reference restatement
(oracle/torch_ref.py) and (b) central finite differences (h = 1e-3) of that
reference at points whose Wiener gain stays away from its kink.  The forward
of the function is checked against the FP64 reference as well.
"""
import numpy as np
import pytest

from dfttest2_b200.frontend import plugin_arguments
from oracle import torch_ref as TR

pytestmark = pytest.mark.gpu


def _setup(torch, C=2, N=4, H=48, W=64, seed=0, **kw):
    rng = np.random.default_rng(seed)
    clean = np.clip(0.5 + 0.15 * np.sin(np.arange(W) * 0.3)[None, None, None, :] +
                    0.1 * np.cos(np.arange(H) * 0.2)[None, None, :, None], 0, 1) * np.ones((C, N, 1, 1))
    noisy = clean + rng.standard_normal((C, N, H, W)) * 0.05
    args = plugin_arguments(full_sigma=True, **kw)
    return args, torch.tensor(noisy, dtype=torch.float32), torch.tensor(clean, dtype=torch.float32)


def _reference_grads(torch, args, noisy, clean, sigma, device):
    x = noisy.double().to(device).requires_grad_(True)
    s = sigma.double().to(device).requires_grad_(True)
    out = torch.stack([TR.dfttest_clip(x[c], args, sigma=s) for c in range(x.shape[0])])
    loss = ((out - clean.double().to(device)) ** 2).mean()
    loss.backward()
    return out.detach(), x.grad.detach(), s.grad.detach(), loss.item()


@pytest.mark.parametrize("kw", [dict(ftype=0, sigma=3.0, tbsize=3), dict(ftype=0, sigma=2.0, tbsize=1),
                                dict(ftype=4, sigma=1.1, pmin=2.0, pmax=300.0, tbsize=3),
                                dict(ftype=0, f0beta=0.7, sigma=3.0, tbsize=5, swin=2),
                                dict(ftype=0, sigma=3.0, tbsize=3, sbsize=8, sosize=4),
                                dict(ftype=0, sigma=3.0, tbsize=3, sbsize=32, sosize=16)])
def test_gradients_match_fp64_reference(kw, cuda_device):
    import torch

    from dfttest2_b200.autograd import DFTTestModule

    args, noisy, clean = _setup(torch, **kw)
    T, B = 2 * args["radius"] + 1, args["block_size"]
    sigma0 = torch.tensor(args["sigma"], dtype=torch.float32).reshape(T, B, B // 2 + 1)
    mod = DFTTestModule(args, sigma0, device=cuda_device)
    x = noisy.to(cuda_device).requires_grad_(True)
    out = mod(x)
    loss = ((out - clean.to(cuda_device)) ** 2).mean()
    loss.backward()
    ref_out, gx_ref, gs_ref, _ = _reference_grads(torch, args, noisy, clean, sigma0, cuda_device)
    assert (out.detach().double() - ref_out).abs().max().item() < 2e-5
    gx = x.grad.double()
    gs = mod.sigma.grad.double()
    ex = ((gx - gx_ref).norm() / gx_ref.norm()).item()
    es = ((gs - gs_ref).norm() / gs_ref.norm()).item()
    print(f"{kw}: rel err d/dx {ex:.2e}, d/dsigma {es:.2e}")
    assert ex < 1e-3
    assert es < 1e-3


def test_gradients_against_finite_differences(cuda_device):
    import torch

    from dfttest2_b200.autograd import DFTTestModule

    args, noisy, clean = _setup(torch, C=1, N=3, H=40, W=40, seed=3, ftype=0, sigma=3.0, tbsize=3)
    sigma0 = torch.tensor(args["sigma"], dtype=torch.float32).reshape(3, 16, 9)
    mod = DFTTestModule(args, sigma0, device=cuda_device)
    x = noisy.to(cuda_device).requires_grad_(True)
    loss = ((mod(x) - clean.to(cuda_device)) ** 2).sum()
    loss.backward()
    gx = x.grad.cpu().double()
    gs = mod.sigma.grad.cpu().double()

    xd = noisy.double()
    sd = sigma0.double()

    def f(xx, ss):
        return ((TR.dfttest_clip(xx[0], args, sigma=ss) - clean[0].double()) ** 2).sum().item()

    h = 1e-3
    rng = np.random.default_rng(0)
    for _ in range(6):
        c, n, i, j = 0, int(rng.integers(3)), int(rng.integers(4, 36)), int(rng.integers(4, 36))
        e = torch.zeros_like(xd)
        e[c, n, i, j] = h
        fd = (f(xd + e, sd) - f(xd - e, sd)) / (2 * h)
        fd2 = (f(xd + 2 * e, sd) - f(xd - 2 * e, sd)) / (4 * h)
        if abs(fd - fd2) > 1e-3 * max(1.0, abs(fd)):
            continue  # a gain kink inside the stencil
        assert abs(gx[c, n, i, j].item() - fd) <= 2e-3 * max(1.0, abs(fd)), (fd, gx[c, n, i, j].item())
    checked = 0
    for idx in [(0, 1, 1), (1, 2, 2), (0, 3, 4), (2, 5, 3), (1, 0, 2), (0, 2, 1)]:
        e = torch.zeros_like(sd)
        e[idx] = h
        fd = (f(xd, sd + e) - f(xd, sd - e)) / (2 * h)
        fd2 = (f(xd, sd + 2 * e) - f(xd, sd - 2 * e)) / (4 * h)
        if abs(fd - fd2) > 1e-3 * max(1.0, abs(fd)):
            continue
        assert abs(gs[idx].item() - fd) <= 2e-3 * max(1.0, abs(fd)), (idx, fd, gs[idx].item())
        checked += 1
    assert checked >= 3


def test_autograd_config_shape_and_timing(cuda_device):
    """8 clips of 256x256 x 9 frames, sigma (3, 16, 9) = 0.05, MSE to clean:
    gradients vs the FP64 reference, forward+backward time vs forward."""
    import torch

    from dfttest2_b200.autograd import DFTTestModule

    args, noisy, clean = _setup(torch, C=8, N=9, H=256, W=256, seed=5, ftype=0, sigma=0.05, tbsize=3)
    mod = DFTTestModule(args, 0.05, device=cuda_device)
    x = noisy.to(cuda_device).requires_grad_(True)
    cl = clean.to(cuda_device)

    def fwd():
        return ((mod(x) - cl) ** 2).mean()

    loss = fwd()
    loss.backward()
    ref_out, gx_ref, gs_ref, _ = _reference_grads(torch, args, noisy, clean, mod.sigma.detach().cpu(), cuda_device)
    ex = ((x.grad.double() - gx_ref).norm() / gx_ref.norm()).item()
    es = ((mod.sigma.grad.double() - gs_ref).norm() / gs_ref.norm()).item()
    assert ex < 1e-3 and es < 1e-3, (ex, es)

    for _ in range(2):
        fwd().backward()
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    e[0].record()
    for _ in range(5):
        with torch.no_grad():
            mod(x)
    e[1].record()
    for _ in range(5):
        x.grad = None
        fwd().backward()
    e[2].record()
    torch.cuda.synchronize()
    t_f = e[0].elapsed_time(e[1]) / 5
    t_fb = e[1].elapsed_time(e[2]) / 5
    print(f"config 4: forward {t_f:.3f} ms, forward+backward {t_fb:.3f} ms, ratio {t_fb / t_f:.2f}; "
          f"rel err d/dx {ex:.2e} d/dsigma {es:.2e}")
