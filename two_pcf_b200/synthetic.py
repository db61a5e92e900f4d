"""Seeded synthetic catalogues with the shapes of the benchmark configurations.

No public dataset is involved: the reference ships no example data.  These
generators produce the inputs the engine is measured and tested on:

* ``box_catalogue``: Neyman-Scott clustered points in a periodic cube plus
  uniform randoms (cartesian input, unit weights, no jackknife);
* ``survey_catalogue``: an equatorial slab (ra in [0, 60] deg, dec in
  [-10, 10] deg uniform in sin(dec), z ~ N(0.3, 0.08) truncated to
  [0.1, 0.5]) with Neyman-Scott clustering in comoving space, lognormal
  weights and a 10 x 10 ra/dec jackknife grid;
* ``bitwise_masks``: inverse-p selection masks (n_runs bits per object set
  independently with probability p_i).

Everything is numpy with a fixed PCG64 seed.  The coordinates are produced
here in double precision; the engine consumes them as given.
"""
from __future__ import annotations

import numpy as np

C_KMS = 299792.458


def comoving_table(omega_m: float = 0.25, h: float = 1.0, z_max: float = 1.0, n: int = 20001):
    """(z, d_c) table of a flat LCDM cosmology in Mpc/h (trapezoid rule)."""
    z = np.linspace(0.0, z_max, n)
    e = 1.0 / np.sqrt(omega_m * (1 + z) ** 3 + (1 - omega_m))
    d = np.concatenate([[0.0], np.cumsum(0.5 * (e[1:] + e[:-1]) * np.diff(z))]) * C_KMS / (100.0 * h)
    return z, d


def radec_to_unit(ra_deg, dec_deg):
    """Unit vector as Galaxy::set forms it (src/galaxy.cpp:8-27)."""
    d2r = np.pi / 180.0
    cd = np.cos(d2r * dec_deg)
    return np.stack([cd * np.cos(d2r * ra_deg), cd * np.sin(d2r * ra_deg), np.sin(d2r * dec_deg)], axis=1)


def neyman_scott_box(rng, n: int, box: float, n_centres: int, mean_members: float, sigma: float):
    """Clustered points in [0, box)^3: Poisson(mean) members per centre,
    Gaussian offsets of width sigma, wrapped periodically; exactly n points."""
    pts = []
    have = 0
    while have < n:
        centres = rng.uniform(0.0, box, size=(n_centres, 3))
        k = rng.poisson(mean_members, size=n_centres)
        rep = np.repeat(centres, k, axis=0)
        p = np.mod(rep + rng.normal(0.0, sigma, size=rep.shape), box)
        pts.append(p)
        have += p.shape[0]
    return np.concatenate(pts)[:n]


def _avoid_first_point_max(xyz):
    """The reference's bounding-box scan never tests point 0 against the
    maximum (src/boxes.cpp:37-40); if point 0 holds a maximum the reference
    indexes past its cell table.  Move such a point away from index 0 so the
    reference stays well defined on these inputs."""
    for _ in range(3):
        if not np.any(xyz[0] >= xyz.max(axis=0)):
            break
        xyz[[0, 1 + np.argmin(xyz[1:, 0])]] = xyz[[1 + np.argmin(xyz[1:, 0]), 0]]
    return xyz


def box_catalogue(seed: int = 1, n_data: int = 100_000, n_rand: int = 300_000, box: float = 500.0,
                  n_centres: int = 2000, mean_members: float = 50.0, sigma: float = 5.0, offset: float = 0.0):
    rng = np.random.default_rng(seed)
    data = neyman_scott_box(rng, n_data, box, n_centres, mean_members, sigma) + offset
    rand = rng.uniform(0.0, box, size=(n_rand, 3)) + offset
    return {"data": {"xyz": _avoid_first_point_max(data)}, "rand": {"xyz": _avoid_first_point_max(rand)}}


def _survey_points(rng, n, z_tab, d_tab, ra_max=60.0, dec_lim=10.0, z_mu=0.3, z_sd=0.08, z_lo=0.1, z_hi=0.5):
    ra = rng.uniform(0.0, ra_max, n)
    s = rng.uniform(np.sin(np.radians(-dec_lim)), np.sin(np.radians(dec_lim)), n)
    dec = np.degrees(np.arcsin(s))
    z = np.empty(0)
    while z.size < n:
        t = rng.normal(z_mu, z_sd, 2 * n)
        z = np.concatenate([z, t[(t >= z_lo) & (t <= z_hi)]])
    z = z[:n]
    return ra, dec, z


def survey_catalogue(seed: int = 2, n_data: int = 1_000_000, n_rand: int = 5_000_000, n_jk_ra: int = 10,
                     n_jk_dec: int = 10, weights: bool = True, cluster_frac: float = 1.0, mean_members: float = 20.0,
                     sigma: float = 5.0, omega_m: float = 0.25, h: float = 1.0):
    """Equatorial slab; returns dict(data=..., rand=...) with ra, dec, z, xyz,
    x_norm, d_comov, weight (float32) and jk (int32) per catalogue."""
    rng = np.random.default_rng(seed)
    z_tab, d_tab = comoving_table(omega_m, h)

    def finish(ra, dec, z, w):
        d = np.interp(z, z_tab, d_tab)
        u = radec_to_unit(ra, dec)
        jk_ra = np.minimum((ra / (60.0 / n_jk_ra)).astype(np.int32), n_jk_ra - 1)
        jk_dec = np.minimum(((dec + 10.0) / (20.0 / n_jk_dec)).astype(np.int32), n_jk_dec - 1)
        return {"ra": ra, "dec": dec, "z": z, "d_comov": d, "x_norm": u, "xyz": u * d[:, None],
                "weight": w, "jk": (jk_ra * n_jk_dec + jk_dec).astype(np.int32)}

    # data: Neyman-Scott in comoving space around centres drawn from the selection
    n_cl = int(n_data * cluster_frac)
    parts_ra, parts_dec, parts_z = [], [], []
    have = 0
    while have < n_cl:
        nc = max(1, int((n_cl - have) / mean_members * 1.3))
        cra, cdec, cz = _survey_points(rng, nc, z_tab, d_tab)
        cxyz = radec_to_unit(cra, cdec) * np.interp(cz, z_tab, d_tab)[:, None]
        k = rng.poisson(mean_members, nc)
        m = np.repeat(cxyz, k, axis=0) + rng.normal(0.0, sigma, (int(k.sum()), 3))
        dist = np.linalg.norm(m, axis=1)
        ra = np.degrees(np.arctan2(m[:, 1], m[:, 0])) % 360.0
        dec = np.degrees(np.arcsin(np.clip(m[:, 2] / dist, -1, 1)))
        z = np.interp(dist, d_tab, z_tab)
        keep = (ra < 60.0) & (np.abs(dec) < 10.0) & (z >= 0.1) & (z <= 0.5)
        parts_ra.append(ra[keep])
        parts_dec.append(dec[keep])
        parts_z.append(z[keep])
        have += int(keep.sum())
    ra = np.concatenate(parts_ra)[:n_cl]
    dec = np.concatenate(parts_dec)[:n_cl]
    z = np.concatenate(parts_z)[:n_cl]
    if n_cl < n_data:
        r2, d2, z2 = _survey_points(rng, n_data - n_cl, z_tab, d_tab)
        ra, dec, z = np.concatenate([ra, r2]), np.concatenate([dec, d2]), np.concatenate([z, z2])
    perm = rng.permutation(n_data)
    ra, dec, z = ra[perm], dec[perm], z[perm]
    wd = rng.lognormal(0.0, 0.2, n_data).astype(np.float32) if weights else np.ones(n_data, np.float32)
    data = finish(ra, dec, z, wd)
    rra, rdec, rz = _survey_points(rng, n_rand, z_tab, d_tab)
    wr = rng.lognormal(0.0, 0.2, n_rand).astype(np.float32) if weights else np.ones(n_rand, np.float32)
    rand = finish(rra, rdec, rz, wr)
    return {"data": data, "rand": rand, "n_jk": n_jk_ra * n_jk_dec}


def bitwise_masks(seed: int, n: int, n_runs: int = 2048, n_mask_ints: int = 32, p_lo: float = 0.3,
                  p_hi: float = 1.0, all_set: bool = False):
    """Signed int64 masks, object-major (n, n_mask_ints); bit b of the run
    index is set with probability p_i.  all_set=True gives every bit set."""
    if all_set:
        return np.full((n, n_mask_ints), -1, dtype=np.int64)
    rng = np.random.default_rng(seed)
    p = rng.uniform(p_lo, p_hi, n)
    out = np.zeros((n, n_mask_ints), dtype=np.uint64)
    for m in range(n_mask_ints):
        bits = rng.random((n, 64)) < p[:, None]
        nb = max(0, min(64, n_runs - 64 * m))
        bits[:, nb:] = False
        out[:, m] = np.packbits(bits, axis=1, bitorder="little").view(np.uint64).ravel()
    return out.view(np.int64)
