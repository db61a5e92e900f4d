"""Weight gradients through the adjoint kernel (tpcf_count_backward) and its
torch.autograd binding, on a small version of the weight-gradient workload:
w = exp(theta . f) with smooth per-object features f, loss = sum over s-mu
bins of (xi - xi_target)^2.

Checked against
  * the oracle's FP64 CPU adjoint of the same pair sums (orc_count_backward),
  * a complete FP64 CPU gradient (oracle pair sums and adjoint, the
    normalisation and Landy-Szalay chain in numpy),
  * central finite differences of the GPU loss in the per-object weights,
    1e-6 relative: the weights sit on a 2^-8 grid and the step is 2^-8, so
    every float pair product (the reference's w1 * w2 in float) is exact and
    the loss is the smooth function the gradient describes;
  * central finite differences in theta (Richardson-extrapolated steps of
    2e-3 and 1e-3; a plain step of 1e-6 would drown in the float rounding of
    each w = exp(theta . f)): 3e-6 of the gradient's scale (measured ~1.3e-6,
    the rounding noise of the float weights)."""
import numpy as np
import pytest

import two_pcf_b200 as tp
from oracle import port
from two_pcf_b200 import synthetic

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

AX1, AX2 = (10.0, 60.0, 1.0, 10), (0.0, 1.0, 0.0, 5)  # every bin well filled by the randoms
OAXES = AX1 + AX2


def sky_points(seed, n, clustered):
    rng = np.random.default_rng(seed)
    if clustered:
        nc = n // 25
        ra_c = rng.uniform(1, 19, nc)
        dec_c = rng.uniform(-4, 4, nc)
        d_c = rng.uniform(420, 680, nc)
        ra = np.repeat(ra_c, 25)[:n] + rng.normal(0, 0.3, n)
        dec = np.repeat(dec_c, 25)[:n] + rng.normal(0, 0.3, n)
        d = np.repeat(d_c, 25)[:n] + rng.normal(0, 3.0, n)
    else:
        ra = rng.uniform(0, 20, n)
        dec = np.degrees(np.arcsin(rng.uniform(np.sin(np.radians(-5)), np.sin(np.radians(5)), n)))
        d = rng.uniform(400, 700, n)
    u = synthetic.radec_to_unit(ra, dec)
    return {"xyz": u * d[:, None], "unit": u, "dcom": d, "ra": ra, "dec": dec}


def features(c, seed, k=8):
    """Smooth random Fourier fields over ra/dec, standardised."""
    rng = np.random.default_rng(seed)
    f = np.empty((c["ra"].size, k))
    for j in range(k):
        a, b, ph = rng.normal(0, 0.3, 2).tolist() + [rng.uniform(0, 2 * np.pi)]
        f[:, j] = np.cos(a * c["ra"] + b * c["dec"] + ph)
    return (f - f.mean(0)) / f.std(0)


@pytest.fixture(scope="module")
def setup(ctx):
    d = sky_points(1, 2500, True)
    r = sky_points(2, 6000, False)
    t = sky_points(3, 2500, True)
    D = tp.Catalog(ctx, d["xyz"], d["unit"], d["dcom"], np.ones(2500, np.float32))
    R = tp.Catalog(ctx, r["xyz"], r["unit"], r["dcom"], np.ones(6000, np.float32))
    T = tp.Catalog(ctx, t["xyz"], t["unit"], t["dcom"])
    b = tp.Binning(ctx, tp.S_MU, AX1, AX2)
    # target xi: an independent clustered catalogue with unit weights
    dd, _, _ = tp.count(ctx, T, None, b)
    dr, _, _ = tp.count(ctx, T, R, b)
    rr, _, _ = tp.count(ctx, R, None, b)
    nd = 2 * dd / (2500.0 ** 2 * (1 - 1 / 2500))
    ndr = dr / (2500.0 * 6000.0)
    nr = 2 * rr / (6000.0 ** 2 * (1 - 1 / 6000))
    xi_t = np.where(nr > 0, (nd - 2 * ndr) / np.where(nr > 0, nr, 1) + 1, 0.0)
    return {"d": d, "r": r, "D": D, "R": R, "b": b, "xi_t": xi_t, "fd": features(d, 11), "fr": features(r, 12)}


def torch_loss(ctx, s, wd, wr, precision=tp.FP32_GUARD):
    from two_pcf_b200.autograd import pair_counts
    D, R, b = s["D"], s["R"], s["b"]
    # Galaxy::weight is float: round, passing the gradient straight through
    wd = wd + (wd.to(torch.float32).to(torch.float64) - wd).detach()
    wr = wr + (wr.to(torch.float32).to(torch.float64) - wr).detach()
    dd = pair_counts(wd, None, ctx, D, None, b, precision)
    dr = pair_counts(wd, wr, ctx, D, R, b, precision)
    rr = pair_counts(wr, None, ctx, R, None, b, precision)
    nd_, nr_ = wd.numel(), wr.numel()
    sd, sr = wd.sum(), wr.sum()
    # JKHists::normalise (src/hist.cpp:290-367) of the doubled auto counts
    ndd = 2 * dd / (sd * sd * (1 - 1.0 / nd_))
    ndr = dr / (sd * sr)
    nrr = 2 * rr / (sr * sr * (1 - 1.0 / nr_))
    ok = nrr > 0
    xi = torch.where(ok, (ndd - 2 * ndr) / torch.where(ok, nrr, torch.ones_like(nrr)) + 1, torch.zeros_like(nrr))
    t = torch.from_numpy(s["xi_t"])
    return ((xi - t) ** 2).sum()


def cpu_loss_and_grad(s, wd, wr):
    """FP64 CPU loss and dL/dw: oracle pair sums and adjoint, normalisation
    and xi chain in numpy."""
    d, r = s["d"], s["r"]
    cd = port.Cat(d["xyz"], unit=d["unit"], dcom=d["dcom"], w=wd.astype(np.float32))
    cr = port.Cat(r["xyz"], unit=r["unit"], dcom=r["dcom"], w=wr.astype(np.float32))
    f_dd, _, _ = port.count_3d(port.S_MU, cd, None, is_auto=True, axes=OAXES)
    f_dr, _, _ = port.count_3d(port.S_MU, cd, cr, is_auto=False, axes=OAXES)
    f_rr, _, _ = port.count_3d(port.S_MU, cr, None, is_auto=True, axes=OAXES)
    w32d, w32r = wd.astype(np.float32).astype(np.float64), wr.astype(np.float32).astype(np.float64)
    # the normalisation uses the float weights summed in double
    sd, sr = w32d.sum(), w32r.sum()
    n1, n2 = wd.size, wr.size
    kd, kr = sd * sd * (1 - 1 / n1), sr * sr * (1 - 1 / n2)
    ndd, ndr, nrr = f_dd / kd, f_dr / (sd * sr), f_rr / kr
    ok = nrr > 0
    xi = np.where(ok, (ndd - 2 * ndr) / np.where(ok, nrr, 1) + 1, 0.0)
    L = float(((xi - s["xi_t"]) ** 2).sum())
    gx = np.where(ok, 2 * (xi - s["xi_t"]), 0.0)
    safe = np.where(ok, nrr, 1)
    g_ndd, g_ndr, g_nrr = gx / safe, -2 * gx / safe, -gx * (ndd - 2 * ndr) / safe ** 2
    # raw (unordered) sums: f_dd = 2 * raw
    G_dd, G_dr, G_rr = 2 * g_ndd / kd, g_ndr / (sd * sr), 2 * g_nrr / kr
    gd1, _ = port.count_backward(port.S_MU, cd, None, is_auto=True, axes=OAXES, G=G_dd)
    gd2, gr2 = port.count_backward(port.S_MU, cd, cr, is_auto=False, axes=OAXES, G=G_dr)
    gr1, _ = port.count_backward(port.S_MU, cr, None, is_auto=True, axes=OAXES, G=G_rr)
    gd = gd1 + gd2 + (-2 * (g_ndd * ndd).sum() / sd - (g_ndr * ndr).sum() / sd)
    gr = gr1 + gr2 + (-2 * (g_nrr * nrr).sum() / sr - (g_ndr * ndr).sum() / sr)
    return L, gd, gr


@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64])
@pytest.mark.parametrize("auto", [True, False])
def test_backward_matches_oracle_adjoint(ctx, setup, auto, precision):
    s = setup
    rng = np.random.default_rng(4)
    wd = rng.lognormal(0, 0.3, 2500).astype(np.float32)
    wr = rng.lognormal(0, 0.3, 6000).astype(np.float32)
    s["D"].set_weights(wd)
    s["R"].set_weights(wr)
    G = rng.normal(size=s["b"].nb)
    ga, gb, st = tp.count_backward(ctx, s["D"], None if auto else s["R"], s["b"], G, precision)
    cd = port.Cat(s["d"]["xyz"], unit=s["d"]["unit"], dcom=s["d"]["dcom"], w=wd)
    cr = port.Cat(s["r"]["xyz"], unit=s["r"]["unit"], dcom=s["r"]["dcom"], w=wr)
    oa, ob = port.count_backward(port.S_MU, cd, None if auto else cr, is_auto=auto, axes=OAXES, G=G)
    assert np.abs(oa).max() > 0
    scale = np.abs(G).max() * float(wd.max()) * 1e-12
    np.testing.assert_allclose(ga, oa, rtol=1e-11, atol=scale * 100)
    if not auto:
        np.testing.assert_allclose(gb, ob, rtol=1e-11, atol=scale * 100)
    assert st["in_range"] > 0


def test_backward_rejects_nonfinite_histogram_gradient(ctx, setup):
    """The gradient terms are summed in fixed point scaled by max|dL/dfull|:
    a non-finite entry is refused before any launch."""
    s = setup
    G = np.ones(s["b"].nb)
    G[3] = np.nan
    with pytest.raises(tp.TpcfError):
        tp.count_backward(ctx, s["D"], None, s["b"], G)
    G[3] = np.inf
    with pytest.raises(tp.TpcfError):
        tp.count_backward(ctx, s["D"], s["R"], s["b"], G)


def test_weight_gradient_vs_fp64_cpu_and_finite_differences(ctx, setup):
    s = setup
    rng = np.random.default_rng(5)
    theta = torch.tensor(rng.normal(0, 0.05, 8), dtype=torch.float64, requires_grad=True)
    Fd, Fr = torch.from_numpy(s["fd"]), torch.from_numpy(s["fr"])
    wd = torch.exp(Fd @ theta)
    wr = torch.exp(Fr @ theta)
    wd.retain_grad()
    wr.retain_grad()
    L = torch_loss(ctx, s, wd, wr)
    L.backward()
    gth = theta.grad.numpy().copy()
    gwd, gwr = wd.grad.numpy().copy(), wr.grad.numpy().copy()

    # FP64 CPU gradient of the same loss at the same (float) weights
    wd_np, wr_np = wd.detach().numpy(), wr.detach().numpy()
    Lc, gdc, grc = cpu_loss_and_grad(s, wd_np, wr_np)
    assert abs(L.item() - Lc) <= 1e-9 * abs(Lc)
    np.testing.assert_allclose(gwd, gdc, rtol=1e-8, atol=1e-8 * np.abs(gdc).max())
    np.testing.assert_allclose(gwr, grc, rtol=1e-8, atol=1e-8 * np.abs(grc).max())

    # central differences in single weights, on a 2^-8 grid with a 2^-8 step:
    # every pair product is exact in float
    w32d = (np.round(wd_np * 256) / 256).astype(np.float32)
    w32r = (np.round(wr_np * 256) / 256).astype(np.float32)
    with torch.enable_grad():
        vd = torch.from_numpy(w32d.astype(np.float64)).requires_grad_(True)
        vr = torch.from_numpy(w32r.astype(np.float64)).requires_grad_(True)
        torch_loss(ctx, s, vd, vr).backward()
    gwd, gwr = vd.grad.numpy(), vr.grad.numpy()

    def loss_at(vd, vr):
        with torch.no_grad():
            return torch_loss(ctx, s, torch.from_numpy(vd.astype(np.float64)),
                              torch.from_numpy(vr.astype(np.float64))).item()

    for which, idx in (("d", 17), ("d", 1203), ("r", 40), ("r", 5000)):
        base = w32d if which == "d" else w32r
        h = np.float32(2.0 ** -8)
        up, dn = base.copy(), base.copy()
        up[idx] += h
        dn[idx] -= h
        if which == "d":
            fd = (loss_at(up, w32r) - loss_at(dn, w32r)) / (2 * float(h))
            an = gwd[idx]
        else:
            fd = (loss_at(w32d, up) - loss_at(w32d, dn)) / (2 * float(h))
            an = gwr[idx]
        assert abs(fd - an) <= 1e-6 * abs(an) + 1e-9 * np.abs(gwd).max(), (which, idx, fd, an)

    # central differences in theta, Richardson-extrapolated (steps 2e-3 and
    # 1e-3): the step error drops to O(h^4) while the float-rounding noise of
    # the weights stays ~1e-7 of the gradient
    th0 = theta.detach().numpy()

    def loss_theta(th):
        with torch.no_grad():
            tt = torch.from_numpy(th)
            return torch_loss(ctx, s, torch.exp(Fd @ tt), torch.exp(Fr @ tt)).item()

    for k in range(8):
        d = []
        for h in (2e-3, 1e-3):
            e = np.zeros(8)
            e[k] = h
            d.append((loss_theta(th0 + e) - loss_theta(th0 - e)) / (2 * h))
        fd = (4 * d[1] - d[0]) / 3
        assert abs(fd - gth[k]) <= 3e-6 * np.abs(gth).max(), (k, fd, gth[k], d)


def test_theta_chain_rule_at_fixed_float_weights(ctx, setup):
    """dL/dtheta at the spec's tolerance, apart from the float rounding of
    the weights: the weights are held at their float values, dL/dw comes from
    the FP64 CPU gradient (oracle pair sums and adjoint), dw/dtheta from
    central differences with step 1e-6 of w = exp(theta . f) in double, and
    sum_i dL/dw_i dw_i/dtheta must equal the GPU's dL/dtheta (autograd through
    the adjoint kernel) to 1e-6 relative."""
    s = setup
    rng = np.random.default_rng(6)
    theta = torch.tensor(rng.normal(0, 0.05, 8), dtype=torch.float64, requires_grad=True)
    Fd, Fr = torch.from_numpy(s["fd"]), torch.from_numpy(s["fr"])
    wd = torch.exp(Fd @ theta)
    wr = torch.exp(Fr @ theta)
    torch_loss(ctx, s, wd, wr).backward()
    g_gpu = theta.grad.numpy().copy()
    w32d = wd.detach().numpy().astype(np.float32).astype(np.float64)
    w32r = wr.detach().numpy().astype(np.float32).astype(np.float64)
    _, gdc, grc = cpu_loss_and_grad(s, w32d, w32r)
    th0, h = theta.detach().numpy(), 1e-6
    chain = np.empty(8)
    for k in range(8):
        e = np.zeros(8)
        e[k] = h
        dwd = (np.exp(s["fd"] @ (th0 + e)) - np.exp(s["fd"] @ (th0 - e))) / (2 * h)
        dwr = (np.exp(s["fr"] @ (th0 + e)) - np.exp(s["fr"] @ (th0 - e))) / (2 * h)
        chain[k] = gdc @ dwd + grc @ dwr
    np.testing.assert_allclose(g_gpu, chain, rtol=1e-6, atol=1e-6 * np.abs(chain).max())
