"""Seeded synthetic particle sets standing in for the reference's inputs.

The reference reads Fortran-unformatted particle files (src/reader.f90:410-465:
positions in cMpc inside [-L/2, L/2], velocities in km/s, masses in Msun).  No
public dataset is used here; the generators below reproduce the shapes, sizes and
value distributions of the benchmark workloads:

  * ``mock_spheres``   -- Poisson-uniform box with underdense spheres and a radial
                          outflow inside them (64^3, 2^18 particles, L=100);
  * ``lognormal``      -- particles Poisson-sampled from exp(G) of a Gaussian random
                          field with P(k) ~ k^n, velocities from linear theory
                          (v ~ grad(phi), scaled to a target rms).

``to_reader_units`` applies the unit conversion READ_BINARY_PART_1 performs
(src/reader.f90:455-458) so the arrays can be passed to the C-ABI.
"""
from __future__ import annotations

import numpy as np

from ._abi import UM, UV

RHO_CRIT_H2 = 2.775e11      # critical density / h^2 [Msun / Mpc^3]


def _mean_mass(n, box, ache=0.678, omega0=0.31):
    rho = omega0 * RHO_CRIT_H2 * ache ** 2
    return np.float32(rho * box ** 3 / n)


def mock_spheres(n=2 ** 18, box=100.0, nsph=8, rmin=5.0, rmax=15.0, contrast=0.2,
                 sigma_v=300.0, outflow=0.3, ache=0.678, seed=1001):
    """Uniform box with ``nsph`` non-overlapping spheres at ``contrast`` x mean
    density; velocities N(0, sigma_v) plus outflow*H0*r inside each sphere."""
    rng = np.random.default_rng(seed)
    half = box / 2.0
    cen, rad = [], []
    while len(cen) < nsph:
        r = rng.uniform(rmin, rmax)
        c = rng.uniform(-half + r, half - r, 3)
        if all(np.linalg.norm(c - c2) > r + r2 for c2, r2 in zip(cen, rad)):
            cen.append(c)
            rad.append(r)
    cen = np.array(cen)
    rad = np.array(rad)
    pos = np.empty((0, 3))
    while len(pos) < n:
        cand = rng.uniform(-half, half, (2 * (n - len(pos)) + 1024, 3))
        d = np.linalg.norm(cand[:, None, :] - cen[None], axis=2)
        inside = (d < rad[None]).any(1)
        keep = ~inside | (rng.random(len(cand)) < contrast)
        pos = np.concatenate([pos, cand[keep]])
    pos = pos[:n]
    vel = rng.normal(0.0, sigma_v, (n, 3))
    h0 = 100.0 * ache
    d = pos[:, None, :] - cen[None]
    dn = np.linalg.norm(d, axis=2)
    for s in range(nsph):
        m = dn[:, s] < rad[s]
        vel[m] += outflow * h0 * d[m, s]
    m = np.full(n, _mean_mass(n, box, ache), np.float32)
    pos = np.clip(pos, -half, half).astype(np.float32)
    vel = vel.astype(np.float32)
    return dict(x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(),
                vx=vel[:, 0].copy(), vy=vel[:, 1].copy(), vz=vel[:, 2].copy(), m=m,
                centres=cen.astype(np.float32), radii=rad.astype(np.float32), box=box)


def _grf(ng, box, index, sigma, rng):
    """Gaussian random field on ng^3 with P(k) ~ k^index, unit-normalised to sigma;
    returns the field and its linear-theory velocity direction fields."""
    kx = np.fft.fftfreq(ng, d=box / ng) * 2 * np.pi
    kz = np.fft.rfftfreq(ng, d=box / ng) * 2 * np.pi
    KX, KY, KZ = np.meshgrid(kx, kx, kz, indexing="ij")
    k2 = KX ** 2 + KY ** 2 + KZ ** 2
    k2[0, 0, 0] = 1.0
    amp = np.sqrt(k2 ** (index / 2.0))
    amp[0, 0, 0] = 0.0
    noise = rng.normal(size=(ng, ng, ng))
    dk = np.fft.rfftn(noise) * amp
    g = np.fft.irfftn(dk, s=(ng, ng, ng))
    scale = sigma / g.std()
    g *= scale
    dk *= scale
    # linear theory: div v ~ -delta  =>  v_k = i k delta_k / k^2
    vel = [np.fft.irfftn(1j * K * dk / k2, s=(ng, ng, ng)) for K in (KX, KY, KZ)]
    return g, vel


def lognormal(n=2 ** 24, ng=256, box=250.0, index=-1.5, sigma_ln=1.0, vrms=350.0,
              bias=1.0, ache=0.678, seed=1002):
    """Particles Poisson-sampled from a lognormal field exp(bias*G - ...), with
    linear-theory velocities scaled to ``vrms``; axes indexed (x, y, z)."""
    rng = np.random.default_rng(seed)
    g, vel = _grf(ng, box, index, sigma_ln, rng)
    rho = np.exp(bias * g)
    p = rho.ravel() / rho.sum()
    cdf = np.cumsum(p)
    cdf[-1] = 1.0
    cell = np.searchsorted(cdf, rng.random(n), side="right")
    cell = np.minimum(cell, ng ** 3 - 1)
    ix, iy, iz = np.unravel_index(cell, (ng, ng, ng))
    h = box / ng
    off = rng.random((n, 3))
    x = (-box / 2 + (ix + off[:, 0]) * h)
    y = (-box / 2 + (iy + off[:, 1]) * h)
    z = (-box / 2 + (iz + off[:, 2]) * h)
    v = np.stack([vf.ravel()[cell] for vf in vel], 1)
    v *= vrms / np.sqrt((v ** 2).sum(1).mean())
    half = box / 2
    pos = np.clip(np.stack([x, y, z], 1), -half, half).astype(np.float32)
    v = v.astype(np.float32)
    m = np.full(n, _mean_mass(n, box, ache), np.float32)
    return dict(x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(),
                vx=v[:, 0].copy(), vy=v[:, 1].copy(), vz=v[:, 2].copy(), m=m, box=box)


def lognormal_torch(n, ng, box, index, sigma_ln=1.0, vrms=350.0, ache=0.678, seed=1004,
                    device="cuda"):
    """GPU version of ``lognormal`` for the 512^3 / 2^27 workload (torch is used only
    to make the synthetic input; it plays no part in the measured path)."""
    import torch
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    kx = torch.fft.fftfreq(ng, d=box / ng, device=device) * 2 * np.pi
    kz = torch.fft.rfftfreq(ng, d=box / ng, device=device) * 2 * np.pi
    KX = kx.view(-1, 1, 1)
    KY = kx.view(1, -1, 1)
    KZ = kz.view(1, 1, -1)
    k2 = KX ** 2 + KY ** 2 + KZ ** 2
    k2[0, 0, 0] = 1.0
    amp = k2 ** (index / 4.0)
    amp[0, 0, 0] = 0.0
    noise = torch.randn((ng, ng, ng), generator=gen, device=device)
    dk = torch.fft.rfftn(noise) * amp
    del noise
    g = torch.fft.irfftn(dk, s=(ng, ng, ng))
    scale = sigma_ln / g.std()
    g *= scale
    dk *= scale
    rho = torch.exp(g.double())
    del g
    cdf = torch.cumsum(rho.view(-1) / rho.sum(), 0)
    del rho
    cdf[-1] = 1.0
    u = torch.rand(n, generator=gen, device=device, dtype=torch.float64)
    cell = torch.searchsorted(cdf, u, right=True).clamp_(max=ng ** 3 - 1)
    del cdf, u
    h = box / ng
    iz = cell % ng
    iy = (cell // ng) % ng
    ix = cell // (ng * ng)
    off = torch.rand((n, 3), generator=gen, device=device, dtype=torch.float64)
    half = box / 2
    x = (-half + (ix + off[:, 0]) * h).clamp_(-half, half).float()
    y = (-half + (iy + off[:, 1]) * h).clamp_(-half, half).float()
    z = (-half + (iz + off[:, 2]) * h).clamp_(-half, half).float()
    del off, ix, iy, iz
    vs = []
    for K in (KX, KY, KZ):
        vf = torch.fft.irfftn(1j * K * dk / k2, s=(ng, ng, ng)).view(-1)
        vs.append(vf[cell])
        del vf
    v = torch.stack(vs, 1)
    v *= vrms / v.double().pow(2).sum(1).mean().sqrt().float()
    m = torch.full((n,), float(_mean_mass(n, box, ache)), device=device)
    return dict(x=x, y=y, z=z, vx=v[:, 0].contiguous(), vy=v[:, 1].contiguous(),
                vz=v[:, 2].contiguous(), m=m, box=box)


def to_reader_units(parts: dict) -> dict:
    """masses / UM and velocities / UV in REAL*4, as src/reader.f90:455-458."""
    out = dict(parts)
    mod = np
    try:
        import torch
        if isinstance(parts["m"], torch.Tensor):
            out["m"] = parts["m"] / float(UM)
            for k in ("vx", "vy", "vz"):
                out[k] = parts[k] / float(UV)
            return out
    except ImportError:
        pass
    out["m"] = (mod.asarray(parts["m"], np.float32) / UM).astype(np.float32)
    for k in ("vx", "vy", "vz"):
        out[k] = (mod.asarray(parts[k], np.float32) / UV).astype(np.float32)
    return out
