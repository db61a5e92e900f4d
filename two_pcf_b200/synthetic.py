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


# Footprint and jackknife boundaries as decimal literals (sin 10 deg, tan 60 deg,
# tan(6k deg), sin(-10 + 2k deg)), so that no run-time libm call decides them.
SIN_DEC_LIM = 0.17364817766693033
TAN_RA_MAX = 1.7320508075688772
TAN_RA_EDGES = np.array([0.10510423526567647, 0.21255656167002213, 0.3249196962329063, 0.4452286853085362,
                         0.5773502691896257, 0.7265425280053609, 0.9004040442978399, 1.110612514829193,
                         1.3763819204711734])
SIN_DEC_EDGES = np.array([-0.13917310096006544, -0.10452846326765347, -0.0697564737441253, -0.03489949670250097,
                          0.0, 0.03489949670250097, 0.0697564737441253, 0.10452846326765347, 0.13917310096006544])


def comoving_table(omega_m: float = 0.25, h: float = 1.0, z_max: float = 1.0, n: int = 20001):
    """(z, d_c) table of a flat LCDM cosmology in Mpc/h (trapezoid rule).
    Only correctly rounded operations (+, *, /, sqrt, a sequential cumsum),
    so the table is the same on every x86-64 host."""
    z = np.linspace(0.0, z_max, n)
    a = 1.0 + z
    e = 1.0 / np.sqrt(omega_m * (a * a * a) + (1 - omega_m))
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


def _footprint_directions(rng, n):
    """n unit vectors uniform on the footprint (ra in [0, 60) deg, sin(dec)
    uniform on [-sin 10, sin 10]): the azimuth of a point drawn uniformly in
    the 60-degree sector of the unit disc, the z component drawn uniformly."""
    cs, sn = [], []
    have = 0
    while have < n:
        m = 2 * (n - have) + 64   # the sector is 52 % of the unit square
        a = rng.uniform(0.0, 1.0, m)
        b = rng.uniform(0.0, 1.0, m)
        r2 = a * a + b * b
        ok = (r2 <= 1.0) & (r2 > 1e-4) & (b < TAN_RA_MAX * a)
        rho = np.sqrt(r2[ok])
        cs.append(a[ok] / rho)
        sn.append(b[ok] / rho)
        have += int(ok.sum())
    cphi = np.concatenate(cs)[:n]
    sphi = np.concatenate(sn)[:n]
    uz = rng.uniform(-SIN_DEC_LIM, SIN_DEC_LIM, n)
    c = np.sqrt(1.0 - uz * uz)
    return np.stack([c * cphi, c * sphi, uz], axis=1)


def _redshifts(rng, n, z_mu=0.3, z_sd=0.08, z_lo=0.1, z_hi=0.5):
    z = np.empty(0)
    while z.size < n:
        t = rng.normal(z_mu, z_sd, 2 * n)
        z = np.concatenate([z, t[(t >= z_lo) & (t <= z_hi)]])
    return z[:n]


def survey_catalogue(seed: int = 2, n_data: int = 1_000_000, n_rand: int = 5_000_000, n_jk_ra: int = 10,
                     n_jk_dec: int = 10, weights: bool = True, cluster_frac: float = 1.0, mean_members: float = 20.0,
                     sigma: float = 5.0, omega_m: float = 0.25, h: float = 1.0):
    """Equatorial slab; returns dict(data=..., rand=..., n_jk=...) with
    xyz, x_norm, d_comov, z, weight (float32), jk (int32) and, for reference
    only, ra and dec (degrees) per catalogue.

    Positions and unit vectors are formed from numpy's seeded draws with
    correctly rounded operations only (no vectorised sin, cos, arcsin or
    power, whose SIMD implementations differ between CPUs), so the same seed
    gives bit-identical catalogues on any x86-64 host with this numpy: the
    full-size parity fixtures regenerate their inputs from the seed.  The
    jackknife grid is 10 x 10 regions, 6 deg in ra by 2 deg in dec, defined
    by the literal boundaries above."""
    if (n_jk_ra, n_jk_dec) != (10, 10):
        raise ValueError("the survey footprint's jackknife grid is 10 x 10")
    rng = np.random.default_rng(seed)
    z_tab, d_tab = comoving_table(omega_m, h)
    d_lo, d_hi = np.interp([0.1, 0.5], z_tab, d_tab)

    def finish(u, d, w):
        jk_ra = (u[:, 1][:, None] >= TAN_RA_EDGES[None, :] * u[:, 0][:, None]).sum(1)
        jk_dec = (u[:, 2][:, None] >= SIN_DEC_EDGES[None, :]).sum(1)
        ra = np.degrees(np.arctan2(u[:, 1], u[:, 0]))
        dec = np.degrees(np.arcsin(np.clip(u[:, 2], -1.0, 1.0)))
        return {"ra": ra, "dec": dec, "z": np.interp(d, d_tab, z_tab), "d_comov": d, "x_norm": u,
                "xyz": u * d[:, None], "weight": w, "jk": (jk_ra * n_jk_dec + jk_dec).astype(np.int32)}

    # data: Neyman-Scott in comoving space around centres drawn from the selection
    n_cl = int(n_data * cluster_frac)
    parts_u, parts_d = [], []
    have = 0
    while have < n_cl:
        nc = max(1, int((n_cl - have) / mean_members * 1.3))
        cxyz = _footprint_directions(rng, nc) * np.interp(_redshifts(rng, nc), z_tab, d_tab)[:, None]
        k = rng.poisson(mean_members, nc)
        m = np.repeat(cxyz, k, axis=0) + rng.normal(0.0, sigma, (int(k.sum()), 3))
        dist = np.sqrt(m[:, 0] * m[:, 0] + m[:, 1] * m[:, 1] + m[:, 2] * m[:, 2])
        keep = ((m[:, 0] > 0) & (m[:, 1] >= 0) & (m[:, 1] < TAN_RA_MAX * m[:, 0])
                & (np.abs(m[:, 2]) < SIN_DEC_LIM * dist) & (dist >= d_lo) & (dist <= d_hi))
        parts_u.append(m[keep] / dist[keep][:, None])
        parts_d.append(dist[keep])
        have += int(keep.sum())
    u = np.concatenate(parts_u)[:n_cl]
    d = np.concatenate(parts_d)[:n_cl]
    if n_cl < n_data:
        u2 = _footprint_directions(rng, n_data - n_cl)
        d2 = np.interp(_redshifts(rng, n_data - n_cl), z_tab, d_tab)
        u, d = np.concatenate([u, u2]), np.concatenate([d, d2])
    perm = rng.permutation(n_data)
    u, d = u[perm], d[perm]
    wd = rng.lognormal(0.0, 0.2, n_data).astype(np.float32) if weights else np.ones(n_data, np.float32)
    data = finish(u, d, wd)
    ur = _footprint_directions(rng, n_rand)
    dr = np.interp(_redshifts(rng, n_rand), z_tab, d_tab)
    wr = rng.lognormal(0.0, 0.2, n_rand).astype(np.float32) if weights else np.ones(n_rand, np.float32)
    rand = finish(ur, dr, wr)
    return {"data": data, "rand": rand, "n_jk": n_jk_ra * n_jk_dec}


def catalogue_digest(cat: dict) -> str:
    """sha256 over the arrays that enter a count (xyz, x_norm, d_comov,
    weight, jk) of one catalogue: a fixture made from a seed records it so a
    test can tell whether the seed regenerated the same inputs."""
    import hashlib
    h = hashlib.sha256()
    for k in ("xyz", "x_norm", "d_comov", "weight", "jk"):
        if cat.get(k) is not None:
            h.update(np.ascontiguousarray(cat[k]).tobytes())
    return h.hexdigest()


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
