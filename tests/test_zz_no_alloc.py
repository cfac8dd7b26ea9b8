"""bfpn_idd_noalloc (the integrated depth dose of caller-owned device arrays,
with no allocation by the library) against bfpn_idd of a solver context on
the same state.  The device buffers here belong to the caller (torch tensors);
the entry point only reads and writes them."""
import numpy as np
import pytest

from conftest import golden_config, material_tables
from bfpn_gpu_b200 import Context, capi

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dose_weights(ctx, cfg):
    """(weight of psi^1, weight of psi^2) per group from the context's
    tables: Eq. 24's stopping-power moments plus the catastrophic loss term,
    times dg, over the density."""
    g = cfg.grid()
    p = cfg.phys()
    ng = g.Ng
    dg = g.Lg / ng
    S = ctx.table(capi.TABLE_S_S, ng + 1)
    en = ctx.table(capi.TABLE_EN, ng + 1)
    sig = np.maximum(ctx.table(capi.TABLE_SIGMA_C, ng), 0.0)
    w1 = 0.5 * (S[:-1] + S[1:]) * dg
    w2 = (S[1:] - S[:-1]) / 6.0 * dg
    if p.flags & capi.FLAG_DOSE_CATASTROPHIC_LOSS:
        w1 = w1 + 0.5 * (en[:-1] + en[1:]) * sig * dg
        w2 = w2 + (en[1:] - en[:-1]) * sig * dg / 6.0
    return np.stack([w1, w2], axis=1).reshape(-1) / p.density


def device_state(ctx, dtype):
    return [torch.from_numpy(ctx.get_state(s, c)).to(device="cuda", dtype=dtype) for s in (0, 1) for c in (0, 1)]


def noalloc(cfg, prec, arrays, dc, out, secondary=True):
    F0, f0, F1, f1 = arrays
    stream = torch.cuda.current_stream().cuda_stream
    capi.idd_noalloc(cfg.grid(), prec, cfg.trapezoidal_yz, F0.data_ptr(), f0.data_ptr(),
                     F1.data_ptr() if secondary else None, f1.data_ptr() if secondary else None,
                     dc.data_ptr(), out.data_ptr(), torch.cuda.current_device(), stream)
    torch.cuda.synchronize()
    return out.cpu().numpy().copy()


@pytest.mark.parametrize("prec", [capi.PREC_FP64, capi.PREC_MIXED])
def test_noalloc_matches_context_idd_two_calls(prec):
    cfg = golden_config("8_7")
    mu, sig = material_tables(cfg)
    ctx = Context(cfg.grid(), cfg.phys(), prec)
    ctx.load_tables(mu, sig)
    ctx.init_beam()
    dtype = torch.float64 if prec == capi.PREC_FP64 else torch.float32
    dc = torch.from_numpy(dose_weights(ctx, cfg)).cuda()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    for n_steps in (40, 25):  # two calls in a row, on two different states
        ctx.step(n_steps, fetch=False)
        ref_idd, ref_proxy = ctx.idd()
        arrays = device_state(ctx, dtype)
        got = noalloc(cfg, prec, arrays, dc, out)
        assert ref_idd > 0 and ref_proxy != 0
        assert abs(got[0] - ref_idd) <= 1e-12 * abs(ref_idd)
        # the psi^2 proxy is a signed sum that cancels: its rounding scales with sum |psi^2| dg
        proxy_scale = float(arrays[1].abs().sum()) * cfg.grid().Lg / cfg.ng
        assert abs(got[1] - ref_proxy) <= 1e-12 * proxy_scale
    ctx.close()


def test_noalloc_repeatable_and_primary_only():
    cfg = golden_config("8_7")
    mu, sig = material_tables(cfg)
    ctx = Context(cfg.grid(), cfg.phys(), capi.PREC_FP64)
    ctx.load_tables(mu, sig)
    ctx.init_beam()
    ctx.step(30, fetch=False)
    arrays = device_state(ctx, torch.float64)
    dc = torch.from_numpy(dose_weights(ctx, cfg)).cuda()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    a = noalloc(cfg, capi.PREC_FP64, arrays, dc, out)
    b = noalloc(cfg, capi.PREC_FP64, arrays, dc, out)
    assert np.array_equal(a, b)  # the block partials are summed in a fixed order
    # without the secondary: the proxy is unchanged, the dose drops by the secondary's share
    p = noalloc(cfg, capi.PREC_FP64, arrays, dc, out, secondary=False)
    assert abs(p[1] - a[1]) <= 1e-12 * float(arrays[1].abs().sum()) * cfg.grid().Lg / cfg.ng
    ctx.set_state(1, 0, np.zeros(ctx.cells))
    ctx.set_state(1, 1, np.zeros(ctx.cells))
    ref_idd, _ = ctx.idd()
    assert abs(p[0] - ref_idd) <= 1e-12 * abs(ref_idd)
    ctx.close()


def test_noalloc_rejects_oversized_plane_and_bad_arguments():
    cfg = golden_config("8_7")
    g = cfg.grid()
    big = capi.Grid(Nx=g.Nx, Ny=127, Nz=127, Ng=g.Ng, Nmu=17, Nom=17, Lx=g.Lx, Ly=g.Ly, Lz=g.Lz, Lu=g.Lu, Lv=g.Lv,
                    Lg=g.Lg)  # 128 * 128 * 289 lanes > 4096 * 1024
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    with pytest.raises(capi.BfpnError, match="exceeds the 4194304 lanes"):
        capi.idd_noalloc(big, capi.PREC_FP64, False, p, p, None, None, p, p)
    with pytest.raises(capi.BfpnError, match="both secondary arrays"):
        capi.idd_noalloc(g, capi.PREC_FP64, False, p, p, p, None, p, p)
    with pytest.raises(capi.BfpnError, match="null"):
        capi.idd_noalloc(g, capi.PREC_FP64, False, None, p, None, None, p, p)
    with pytest.raises(capi.BfpnError, match="precision"):
        capi.idd_noalloc(g, 7, False, p, p, None, None, p, p)


@pytest.mark.parametrize("ny,nmu,trap", [(40, 12, False), (40, 12, True), (100, 20, True)])
def test_noalloc_large_planes_and_edge_weights(ny, nmu, trap):
    """Planes of a few hundred and of nearly 4096 blocks (101 x 101 x 400 =
    4,080,400 lanes), with and without the trapezoidal yz edge weights, on
    seeded states: the ticket / last-block path against bfpn_idd."""
    from bfpn_gpu_b200 import make_config
    from conftest import table_dir
    from bfpn_gpu_b200 import read_tables

    cfg = make_config(nx=400, ny=ny, nz=ny, nmu=nmu, nom=nmu, ng=6, ly=4.0, lz=4.0, lg=12.0, beam_energy=6.0,
                      sigma_e=1.0, sigma_yz=0.5, material_name="water", trapezoidal_yz=trap)
    mu, sig = read_tables(table_dir("synthetic500"), cfg.ng)
    ctx = Context(cfg.grid(), cfg.phys(), capi.PREC_FP64)
    ctx.load_tables(mu, sig)
    rng = np.random.default_rng(20261203 + ny + nmu + trap)
    for s in (0, 1):
        ctx.set_state(s, 0, rng.random(ctx.cells))
        ctx.set_state(s, 1, rng.normal(0.0, 1e-3, ctx.cells))
    ref_idd, ref_proxy = ctx.idd()
    arrays = device_state(ctx, torch.float64)
    dc = torch.from_numpy(dose_weights(ctx, cfg)).cuda()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    got = noalloc(cfg, capi.PREC_FP64, arrays, dc, out)
    assert abs(got[0] - ref_idd) <= 1e-12 * abs(ref_idd)
    proxy_scale = float(arrays[1].abs().sum()) * cfg.grid().Lg / cfg.ng
    assert abs(got[1] - ref_proxy) <= 1e-12 * proxy_scale
    # a warm call takes no device memory: the free bytes the driver reports do not move
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    again = noalloc(cfg, capi.PREC_FP64, arrays, dc, out)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert np.array_equal(again, got)
    ctx.close()
