"""Seeded synthetic particle sets standing in for the reference's inputs.

The reference reads Fortran-unformatted particle files (src/reader.f90:410-465:
positions in cMpc inside [-L/2, L/2], velocities in km/s, masses in Msun).  No
public dataset is used here; the generators below reproduce the shapes, sizes and
value distributions of the benchmark workloads:

  * ``mock_spheres``   -- Poisson-uniform box with underdense spheres and a radial
                          outflow inside them (64^3, 2^18 particles, L=100);
  * ``lognormal``      -- particles Poisson-sampled from exp(G) of a Gaussian random
                          field with P(k) ~ k^n, velocities from linear theory
                          (v ~ grad(phi), scaled to a target rms);
  * ``weighted_cone``  -- a survey-like tracer catalogue: power-law masses
                          dn/dM ~ M^-1.9, placed by sampling a biased lognormal
                          field inside a cone with radial selection and a
                          random angular mask (non-periodic);
  * ``add_clumps``     -- dense clumps added to a particle set, to reach the
                          reference's rare branches (ball fallback, FILL_H_ZEROS,
                          NORM = 0).

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
    g = np.fft.irfftn(dk, s=(ng, ng, ng), axes=(0, 1, 2))
    scale = sigma / g.std()
    g *= scale
    dk *= scale
    # linear theory: div v ~ -delta  =>  v_k = i k delta_k / k^2
    vel = [np.fft.irfftn(1j * K * dk / k2, s=(ng, ng, ng), axes=(0, 1, 2)) for K in (KX, KY, KZ)]
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


def power_law_masses(n, slope=-1.9, mlo=1e11, mhi=1e15, rng=None):
    """n masses [Msun] with dn/dM ~ M^slope on [mlo, mhi] (inverse CDF)."""
    rng = rng or np.random.default_rng(0)
    a = slope + 1.0
    u = rng.random(n)
    m = (mlo ** a + u * (mhi ** a - mlo ** a)) ** (1.0 / a)
    return m.astype(np.float32)


def weighted_cone(box=1200.0, ng=128, rmax=600.0, half_angle_deg=60.0, rsel=400.0, mask_frac=0.15,
                  n_target=4_000_000, index=-1.2, sigma_ln=1.0, bias=1.5, vrms=350.0, seed=1005):
    """Weighted tracers in a survey cone (non-periodic geometry).

    Positions: a lognormal field exp(G) on ng^3 (P(k) ~ k^index, sigma_ln),
    sampled with weight rho^bias, kept inside the cone of ``half_angle_deg``
    about +z from the origin out to ``rmax``, with the radial selection
    n(r) ~ exp(-(r/rsel)^2) and a seeded angular mask: the cone's sky is cut
    into 24 x 48 (cos theta, phi) pixels and a random ``mask_frac`` of them
    removed.  Masses: dn/dM ~ M^-1.9 on 1e11..1e15 Msun.  Velocities: linear
    theory from the same field, ``vrms`` rms.  About ``n_target`` tracers."""
    rng = np.random.default_rng(seed)
    g, vel = _grf(ng, box, index, sigma_ln, rng)
    w = np.exp(bias * g)
    h = box / ng
    c1 = np.arange(ng) * h - box / 2 + h / 2
    X, Y, Z = np.meshgrid(c1, c1, c1, indexing="ij")
    R = np.sqrt(X ** 2 + Y ** 2 + Z ** 2)
    cost = np.where(R > 0, Z / np.maximum(R, 1e-30), 1.0)
    cmin = np.cos(np.radians(half_angle_deg))
    inside = (R <= rmax) & (cost >= cmin)
    sel = np.exp(-(R / rsel) ** 2) * inside
    dens = (w * sel).ravel()
    p = dens / dens.sum()
    # expected count n_target before the angular mask
    cell = rng.choice(ng ** 3, size=rng.poisson(n_target), p=p)
    ix, iy, iz = np.unravel_index(cell, (ng, ng, ng))
    off = rng.random((len(cell), 3))
    pos = np.stack([ix + off[:, 0], iy + off[:, 1], iz + off[:, 2]], 1) * h - box / 2
    r = np.linalg.norm(pos, axis=1)
    ct = np.where(r > 0, pos[:, 2] / np.maximum(r, 1e-30), 1.0)
    phi = np.arctan2(pos[:, 1], pos[:, 0])
    keep = (r <= rmax) & (ct >= cmin)
    npc, npp = 24, 48
    masked = rng.random(npc * npp) < mask_frac
    pc = np.clip(((ct - cmin) / (1 - cmin) * npc).astype(int), 0, npc - 1)
    pp = np.clip(((phi + np.pi) / (2 * np.pi) * npp).astype(int), 0, npp - 1)
    keep &= ~masked[pc * npp + pp]
    pos, cell = pos[keep], cell[keep]
    v = np.stack([vf.ravel()[cell] for vf in vel], 1)
    v *= vrms / np.sqrt((v ** 2).sum(1).mean())
    half = box / 2
    pos = np.clip(pos, -half, half).astype(np.float32)
    v = v.astype(np.float32)
    m = power_law_masses(len(pos), rng=rng)
    return dict(x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(),
                vx=v[:, 0].copy(), vy=v[:, 1].copy(), vz=v[:, 2].copy(), m=m, box=box,
                pixel_mask=masked.reshape(npc, npp))


def _cone_pixels(pos, cmin, npc, npp):
    r = np.linalg.norm(pos, axis=1)
    ct = np.where(r > 0, pos[:, 2] / np.maximum(r, 1e-30), 1.0)
    phi = np.arctan2(pos[:, 1], pos[:, 0])
    pc = np.clip(((ct - cmin) / (1 - cmin) * npc).astype(int), 0, npc - 1)
    pp = np.clip(((phi + np.pi) / (2 * np.pi) * npp).astype(int), 0, npp - 1)
    return r, ct, pc * npp + pp


def cone_randoms(n, pixel_mask, box=1200.0, rmax=600.0, half_angle_deg=60.0, rsel=400.0, weight=1e12, seed=2005):
    """Randoms of the survey geometry of ``weighted_cone``: uniform in volume
    inside the cone, thinned by the same radial selection exp(-(r/rsel)^2) and
    angular mask (``pixel_mask`` of weighted_cone), all with the same weight
    [Msun].  Returns x, y, z, w."""
    rng = np.random.default_rng(seed)
    cmin = np.cos(np.radians(half_angle_deg))
    npc, npp = pixel_mask.shape
    out = np.empty((0, 3))
    while len(out) < n:
        m = 4 * (n - len(out)) + 1024
        u = rng.random(m)
        r = rmax * u ** (1 / 3)
        ct = cmin + (1 - cmin) * rng.random(m)
        phi = rng.uniform(-np.pi, np.pi, m)
        st = np.sqrt(1 - ct ** 2)
        q = np.stack([r * st * np.cos(phi), r * st * np.sin(phi), r * ct], 1)
        keep = rng.random(m) < np.exp(-(r / rsel) ** 2)
        _, _, pix = _cone_pixels(q, cmin, npc, npp)
        keep &= ~pixel_mask.ravel()[pix]
        out = np.concatenate([out, q[keep]])
    out = np.clip(out[:n], -box / 2, box / 2).astype(np.float32)
    return dict(x=out[:, 0].copy(), y=out[:, 1].copy(), z=out[:, 2].copy(), w=np.full(n, weight, np.float32))


def cone_mask(nx, pixel_mask, box=1200.0, rmax=600.0, half_angle_deg=60.0):
    """The survey mask on an nx^3 grid (column-major, x fastest): 1 for cells
    whose centre lies inside the cone, within rmax and in an unmasked pixel."""
    h = box / nx
    c1 = -box / 2 + h / 2 + np.arange(nx) * h
    Z, Y, X = np.meshgrid(c1, c1, c1, indexing="ij")
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    cmin = np.cos(np.radians(half_angle_deg))
    r, ct, pix = _cone_pixels(pos, cmin, *pixel_mask.shape)
    inside = (r <= rmax) & (ct >= cmin) & ~pixel_mask.ravel()[pix]
    return inside.astype(np.int8)


def add_clumps(parts: dict, centres, radius, count, seed=0):
    """``parts`` with a clump of ``count`` particles uniform in a ball of
    ``radius`` around each centre (velocities of the clump's centre particle,
    masses equal to the set's first mass)."""
    rng = np.random.default_rng(seed)
    out = {k: v for k, v in parts.items()}
    add = {k: [] for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    for c in np.asarray(centres, np.float64):
        u = rng.normal(size=(count, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        rr = radius * rng.random(count) ** (1 / 3)
        q = c[None] + u * rr[:, None]
        for a, k in enumerate(("x", "y", "z")):
            add[k].append(q[:, a].astype(np.float32))
        for k in ("vx", "vy", "vz"):
            add[k].append(rng.normal(0, np.std(parts[k]), count).astype(np.float32))
        add["m"].append(np.full(count, parts["m"][0], np.float32))
    for k in add:
        out[k] = np.concatenate([np.asarray(parts[k], np.float32)] + add[k])
    return out


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
