"""Seeded synthetic inputs for the holotomography workloads (on the GPU).

The workloads the operator chain is measured on are described by their
sizes and value distributions; no measured dataset is used:

* object: complex refractive-index volume k*dx*(-delta + i beta) made of
  random ellipsoids (semi-axes 5-40 voxels at n = 128, scaled with n;
  centres within radius 50/128 n of the centre, random orientation),
  delta ~ U[1e-7, 1e-6] and beta = delta/50 inside, 0 outside;
* probe: amplitude 1 + 0.1 * Gaussian-smoothed noise (sigma 8 px), phase
  smoothed noise scaled to +-0.3 rad (or a flat unit probe);
* positions: per (angle, distance) shifts uniform in +-amp px;
* data: amplitudes sqrt(Poisson(photons * |forward|^2) / photons).
"""
import math

import numpy as np
import torch


def ellipsoid_phantom(n, nell, seed, wavelength=7.3e-11, voxelsize=20e-9, device="cuda", chunk=64):
    """[n, n, n] complex64 phantom of `nell` random ellipsoids."""
    rng = np.random.default_rng(seed)
    s = n / 128.0
    semi = rng.uniform(5 * s, 40 * s, (nell, 3))
    r = 50 * s * np.cbrt(rng.uniform(0, 1, nell))
    dirs = rng.standard_normal((nell, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    centres = dirs * r[:, None]
    rots = []
    for _ in range(nell):
        q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        rots.append(q)
    delta = rng.uniform(1e-7, 1e-6, nell)
    k = 2 * math.pi / wavelength
    obj = torch.zeros(n, n, n, dtype=torch.complex64, device=device)
    ax = torch.arange(n, device=device, dtype=torch.float32) - n / 2
    yy, xx = torch.meshgrid(ax, ax, indexing="ij")
    for z0 in range(0, n, chunk):
        zz = ax[z0:z0 + chunk][:, None, None].expand(-1, n, n)
        pts = torch.stack([zz, yy.expand_as(zz), xx.expand_as(zz)], dim=-1)
        dl = torch.zeros(zz.shape, device=device)
        for e in range(nell):
            R = torch.as_tensor(rots[e], device=device, dtype=torch.float32)
            c = torch.as_tensor(centres[e], device=device, dtype=torch.float32)
            a = torch.as_tensor(semi[e], device=device, dtype=torch.float32)
            loc = (pts - c) @ R
            inside = ((loc / a) ** 2).sum(-1) <= 1.0
            dl = torch.where(inside, torch.full_like(dl, float(delta[e])), dl)
        obj[z0:z0 + chunk] = (k * voxelsize * torch.complex(-dl, dl / 50)).to(torch.complex64)
    return obj


def _smooth_noise(shape, sigma, gen, device):
    x = torch.randn(*shape, generator=gen, device=device)
    n0, n1 = shape[-2], shape[-1]
    f0 = torch.fft.fftfreq(n0, device=device)[:, None]
    f1 = torch.fft.fftfreq(n1, device=device)[None, :]
    g = torch.exp(-2 * (math.pi * sigma) ** 2 * (f0 ** 2 + f1 ** 2))
    y = torch.fft.ifft2(torch.fft.fft2(x) * g).real
    return y / y.abs().amax(dim=(-2, -1), keepdim=True)


def random_probe(ndist, nz, n, seed, device="cuda", flat=False):
    """[ndist, nz, n] complex64 probe."""
    if flat:
        return torch.ones(ndist, nz, n, dtype=torch.complex64, device=device)
    gen = torch.Generator(device=device).manual_seed(seed)
    amp = 1 + 0.1 * _smooth_noise((ndist, nz, n), 8.0, gen, device)
    ph = 0.3 * _smooth_noise((ndist, nz, n), 8.0, gen, device)
    return torch.polar(amp, ph).to(torch.complex64)


def random_positions(ntheta, ndist, amp, seed, device="cuda"):
    gen = torch.Generator(device=device).manual_seed(seed)
    return (2 * torch.rand(ntheta, ndist, 2, generator=gen, device=device) - 1) * amp


def noisy_amplitudes(amp, photons, seed):
    """sqrt(Poisson(photons |x|^2) / photons) in place of the clean amplitudes."""
    gen = torch.Generator(device=amp.device).manual_seed(seed)
    for i in range(amp.shape[0]):
        inten = torch.poisson(photons * amp[i] ** 2, generator=gen)
        amp[i] = torch.sqrt(inten / photons)
    return amp


def workload_args(n, ntheta, ndist=4, niter=16, distances=(3e-3, 4e-3, 5e-3, 6e-3), wavelength=7.3e-11,
                  voxelsize=20e-9, mask=0.9):
    """Rec arguments of the synthetic workloads: n^3 object, n^2 detector,
    ntheta angles on [0, pi), unit magnification, distances given directly."""
    import types
    return types.SimpleNamespace(
        theta=np.linspace(0, np.pi, ntheta, endpoint=False).astype("float32"), ndist=ndist, ntheta=ntheta,
        nz=n, n=n, nzobj=n, nobj=n, obj_dtype="complex64", mask=mask, lam_prbfit=0.0, rho=[1, 0.05, 0.02],
        niter=niter, nchunk=n, vis_step=-1, err_step=-1, start_iter=0, distance=np.array(distances[:ndist]),
        wavelength=wavelength, voxelsize=voxelsize, norm_magnifications=np.ones(ndist))


def make_problem(n, ntheta, ndist, seed, photons=1e4, device="cuda", pos_amp=2.0, pos_err=0.5, host=False):
    """(args, data, prb0, pos0, truth): a seeded synthetic reconstruction
    problem with noisy amplitudes; the initial state is a zero object, a
    flat probe and perturbed positions.  host=True returns data, prb0 and
    pos0 in pinned host memory (truth stays on the device)."""
    from .rec import Rec
    args = workload_args(n, ntheta, ndist)
    rec = Rec(args)
    obj = ellipsoid_phantom(n, 80 if n >= 512 else 20, seed, device=device)
    prb = random_probe(ndist, n, n, seed + 1, device=device)
    pos = random_positions(ntheta, ndist, pos_amp, seed + 2, device=device)
    data = rec.forward_amplitudes(obj, prb, pos)
    noisy_amplitudes(data, photons, seed + 3)
    gen = torch.Generator(device=device).manual_seed(seed + 4)
    pos0 = pos + pos_err * (2 * torch.rand(pos.shape, generator=gen, device=device) - 1)
    prb0 = torch.ones_like(prb)
    rec.close()
    del rec
    if host:
        data, prb0, pos0 = (t.cpu().pin_memory() for t in (data, prb0, pos0))
    return args, data, prb0, pos0, {"obj": obj, "prb": prb, "pos": pos}
