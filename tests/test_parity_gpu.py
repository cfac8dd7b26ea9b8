"""CUDA path against the oracle, through the C ABI (lib/libbfpn_b200.so).

FP64 mode: every operator and whole depth steps agree with the CPU FP64
restatement to 1e-10 relative (operators 1e-11), on seeded states, and the full
1000-step water 230 MeV runs reproduce the reference's own golden IDD files.
Mixed mode (float state, double energy recursion): operator kernels against
FP64 here; whole-run IDD accuracy at full depth in test_accuracy_gpu.py.
"""
import numpy as np
import pytest

from conftest import golden_config, load_golden, material_tables, rel_err, table_dir
from bfpn_gpu_b200 import Context, capi, make_config, read_tables
from oracle import oracle as O

pytestmark = pytest.mark.gpu

OP_TOL = 1e-11
STEP_TOL = 1e-10


def small_cfg(**kw):
    base = dict(nx=160, ny=6, nz=5, nmu=4, nom=5, ng=40, ly=2.0, lz=1.5, lu=1.0, lv=1.2, lg=59.0, beam_energy=40.0,
                sigma_e=2.0, sigma_yz=0.4, material_name="water", t_final=4.0)
    base.update(kw)
    return make_config(**base)


def build(cfg, tables="synthetic500", precision=capi.PREC_FP64):
    mu, sig = read_tables(table_dir(tables), cfg.ng)
    ctx = Context(cfg.grid(), cfg.phys(), precision)
    ctx.load_tables(mu, sig)
    ctx.init_beam()
    ora = O.Oracle(cfg.grid(), cfg.phys(), mu, sig)
    return ctx, ora


def seeded_states(ctx, seed):
    rng = np.random.default_rng(seed)
    Ng, nyz, NA = ctx.shape
    beam = ctx.table(capi.TABLE_BEAM_YZA, nyz * NA).reshape(nyz, NA)
    e = np.exp(-0.5 * ((np.arange(Ng) - 0.7 * Ng) / (0.1 * Ng)) ** 2)
    F = (e[:, None, None] * (beam / max(beam.max(), 1e-300))[None] + 1e-3 * rng.random((Ng, nyz, NA))).ravel()
    f = 1e-3 * rng.standard_normal(Ng * nyz * NA)
    F1 = 1e-2 * rng.random(Ng * nyz * NA)
    f1 = 1e-3 * rng.standard_normal(Ng * nyz * NA)
    return F, f, F1, f1


def set_both(ctx, ora, states):
    for k, arr in enumerate(states):
        ctx.set_state(k // 2, k % 2, arr)
        ora.set_state(k // 2, k % 2, arr)


def assert_states(ctx, ora, tol, which=((0, 0), (0, 1), (1, 0), (1, 1))):
    for sp, cf in which:
        r = rel_err(ctx.get_state(sp, cf), ora.get_state(sp, cf))
        assert r < tol, ("species", sp, "coef", cf, r)


@pytest.mark.parametrize("flags", [{}, {"legacy_energy": True}, {"eq15_straggling": True},
                                   {"legacy_energy": True, "eq15_straggling": True},
                                   # 225 lanes: rows not a multiple of 16 bytes -> register-prefetch sweep
                                   {"ny": 4, "nz": 4, "nmu": 3, "nom": 3, "eq15_straggling": True}])
def test_energy_operator(flags):
    cfg = small_cfg(**flags)
    ctx, ora = build(cfg)
    set_both(ctx, ora, seeded_states(ctx, 1))
    h = 0.5 * cfg.dt()
    ctx.energy(0, h)
    ora.energy(0, h)
    assert_states(ctx, ora, OP_TOL, ((0, 0), (0, 1)))


def test_secondary_source_and_sourced_energy():
    cfg = small_cfg()
    ctx, ora = build(cfg)
    set_both(ctx, ora, seeded_states(ctx, 2))
    ctx.secondary_source()
    s_gpu = ctx.source()
    s_ora = ora.source()
    assert np.abs(s_ora).max() > 0
    assert rel_err(s_gpu, s_ora) < OP_TOL
    ora.use_direct_source(True)  # the reference's own summation order
    assert rel_err(s_gpu, ora.source()) < OP_TOL
    h = 0.5 * cfg.dt()
    ctx.energy(1, h, with_source=True)
    ora.energy(1, h, with_source=True)
    assert_states(ctx, ora, OP_TOL, ((1, 0), (1, 1)))


@pytest.mark.parametrize("preserve", [False, True])
@pytest.mark.parametrize("shape", [dict(), dict(ny=40, nz=33, nmu=2, nom=3, ng=3)])
def test_transport_operator(preserve, shape):
    cfg = small_cfg(**shape)
    ctx, ora = build(cfg)
    set_both(ctx, ora, seeded_states(ctx, 3))
    for sp, cf in ((0, 0), (0, 1)):
        ctx.transport(sp, cf, 0.5 * cfg.dt(), preserve)
        ora.transport(sp, cf, 0.5 * cfg.dt(), preserve)
    assert_states(ctx, ora, OP_TOL, ((0, 0), (0, 1)))


@pytest.mark.parametrize("preserve", [False, True])
@pytest.mark.parametrize("n,ang", [(4, (3, 3)), (8, (7, 6)), (16, (4, 5)), (32, (3, 2))])
def test_plane_transport_operator(preserve, n, ang):
    """The unrolled whole-plane kernel (square planes) at both angle chunks,
    and the line-walk kernel on the same plane, against the oracle."""
    cfg = small_cfg(ny=n, nz=n, nmu=ang[0], nom=ang[1], ng=6, lz=2.0)
    ctx, ora = build(cfg)
    states = seeded_states(ctx, 6)
    for opt in (1, 8, 0):  # whole plane (4 angles per block), whole plane (8), line walks
        ctx.set_option(capi.OPT_PLANE_TRANSPORT, opt)
        set_both(ctx, ora, states)
        for sp, cf in ((0, 0), (1, 1)):
            ctx.transport(sp, cf, 0.5 * cfg.dt(), preserve)
            ora.transport(sp, cf, 0.5 * cfg.dt(), preserve)
        assert_states(ctx, ora, OP_TOL, ((0, 0), (1, 1)))


@pytest.mark.parametrize("preserve", [False, True])
@pytest.mark.parametrize("ny,nz", [(40, 33), (60, 26), (27, 54)])
def test_tiled_transport_operator(preserve, ny, nz):
    """Planes too large for one block: the unrolled 27 x 27 tile kernel (whole,
    partial and one-cell tiles, both angle chunks) and the line-walk tiles,
    against the oracle."""
    cfg = small_cfg(ny=ny, nz=nz, nmu=3, nom=2, ng=3, ly=4.0, lz=3.0)
    ctx, ora = build(cfg)
    states = seeded_states(ctx, 8)
    for opt in (1, 2, 0):  # unrolled tiles (4 angles per block), unrolled tiles (2), line walks
        ctx.set_option(capi.OPT_PLANE_TRANSPORT, opt)
        set_both(ctx, ora, states)
        for sp, cf in ((0, 0), (1, 1)):
            ctx.transport(sp, cf, 0.5 * cfg.dt(), preserve)
            ora.transport(sp, cf, 0.5 * cfg.dt(), preserve)
        assert_states(ctx, ora, OP_TOL, ((0, 0), (1, 1)))


def test_tiled_transport_mixed_matches_line_walks():
    cfg = small_cfg(ny=80, nz=80, nmu=4, nom=4, ng=2, ly=16.0, lz=16.0)
    ctx, _ = build(cfg, precision=capi.PREC_MIXED)
    states = seeded_states(ctx, 9)
    out = {}
    for opt in (1, 4, 0):
        ctx.set_option(capi.OPT_PLANE_TRANSPORT, opt)
        for k, arr in enumerate(states):
            ctx.set_state(k // 2, k % 2, arr)
        ctx.transport(0, 0, 0.5 * cfg.dt(), False)
        ctx.transport(0, 1, 0.5 * cfg.dt(), True)
        out[opt] = (ctx.get_state(0, 0), ctx.get_state(0, 1))
    for opt in (1, 4):
        for a, b in zip(out[opt], out[0]):
            assert rel_err(a, b) < 2e-6


def test_plane_transport_mixed_matches_line_walks():
    cfg = small_cfg(ny=20, nz=20, nmu=6, nom=7, ng=5, lz=2.0)
    ctx, _ = build(cfg, precision=capi.PREC_MIXED)
    states = seeded_states(ctx, 7)
    out = {}
    for opt in (1, 8, 0):  # whole plane (16 angles per block), whole plane (8), line walks
        for k, arr in enumerate(states):
            ctx.set_state(k // 2, k % 2, arr)
        ctx.transport(0, 0, 0.5 * cfg.dt(), False)
        ctx.transport(0, 1, 0.5 * cfg.dt(), True)
        out[opt] = (ctx.get_state(0, 0), ctx.get_state(0, 1))
    for opt in (1, 8):
        for a, b in zip(out[opt], out[0]):
            assert rel_err(a, b) < 2e-6
    with pytest.raises(capi.BfpnError):
        ctx.set_option(capi.OPT_PLANE_TRANSPORT, 4)  # 4 angles per block is the FP64 chunk


@pytest.mark.parametrize("nom,paired", [(8, True), (6, False)])  # NA 48: pairs share signs; NA 36: pair (2,3) straddles
def test_paired_plane_transport_equals_single_angle_kernel(nom, paired):
    """Two angles per thread on packed fp32x2 (mixed whole-plane transport)
    gives the one-angle kernel's values exactly, including flat regions and
    differences below the limiter's epsilon; where a pair straddles a sign
    change of the direction cosines the one-angle kernel runs."""
    cfg = small_cfg(ny=20, nz=20, nmu=6, nom=nom, ng=5, lz=2.0)
    ctx, _ = build(cfg, precision=capi.PREC_MIXED)
    Ng, nyz, NA = ctx.shape
    states = [a.reshape(Ng, nyz, NA).copy() for a in seeded_states(ctx, 12)]
    for a in states:
        a[1, : nyz // 2] = a[1, 0]                    # flat: zero differences
        a[2] = 3e-11 * np.arange(nyz)[:, None]         # y differences below 1e-10
        a[3, ::7] = 0.0
    out = {}
    for pairs in (1, 0):
        ctx.set_option(capi.OPT_PAIRED_ANGLES, pairs)
        for chunk in (16, 8):
            ctx.set_option(capi.OPT_PLANE_TRANSPORT, chunk)
            for k, arr in enumerate(states):
                ctx.set_state(k // 2, k % 2, arr.ravel())
            ctx.transport(0, 0, 0.5 * cfg.dt(), False)
            ctx.transport(0, 1, 0.5 * cfg.dt(), True)
            ctx.transport(1, 1, 0.37 * cfg.dt(), True)
            out[(pairs, chunk)] = [ctx.get_state(sp, cf) for sp, cf in ((0, 0), (0, 1), (1, 1))]
    for key, got in out.items():
        for a, b in zip(got, out[(0, 16)]):
            assert np.array_equal(a, b), key
    assert np.abs(out[(0, 16)][1]).max() > 0


@pytest.mark.parametrize("n", [8, 20, 7])
def test_paired_dst_equals_one_line_per_thread(n):
    """Mixed-precision angular step: the two-lines-per-thread DST (fp32x2)
    gives the one-line kernel's values exactly (odd N has no pairs)."""
    cfg = small_cfg(ny=5, nz=6, nmu=n, nom=n, ng=7)
    ctx, _ = build(cfg, precision=capi.PREC_MIXED)
    states = seeded_states(ctx, 13)
    out = {}
    for pairs in (1, 0):
        ctx.set_option(capi.OPT_PAIRED_ANGLES, pairs)
        for k, arr in enumerate(states):
            ctx.set_state(k // 2, k % 2, arr)
        ctx.angle(0, 0, cfg.dt())
        ctx.angle(1, 1, 0.3 * cfg.dt())
        out[pairs] = (ctx.get_state(0, 0), ctx.get_state(1, 1))
    for a, b in zip(out[1], out[0]):
        assert np.array_equal(a, b)
    assert not np.array_equal(out[0][0], states[0].astype(np.float32))


def _transport_states(ctx, cfg, seed, opts):
    states = seeded_states(ctx, seed)
    for k, v in opts.items():
        ctx.set_option(k, v)
    for k, arr in enumerate(states):
        ctx.set_state(k // 2, k % 2, arr)
    ctx.transport(0, 0, 0.5 * cfg.dt(), False)
    ctx.transport(0, 1, 0.5 * cfg.dt(), True)
    ctx.transport(1, 0, 0.31 * cfg.dt(), False)
    return [ctx.get_state(sp, cf) for sp, cf in ((0, 0), (0, 1), (1, 0))]


def test_cluster_transport_matches_whole_plane_kernel():
    """Thread-block-cluster transport (2 CTAs holding one 21 x 21 plane, edge
    rows over distributed shared memory) against the whole-plane kernel."""
    cfg = small_cfg(ny=20, nz=20, nmu=6, nom=8, ng=5, lz=2.0)
    ctx, _ = build(cfg, precision=capi.PREC_MIXED)
    a = _transport_states(ctx, cfg, 21, {capi.OPT_STREAM_TRANSPORT: 0, capi.OPT_CLUSTER_TRANSPORT: 2})
    b = _transport_states(ctx, cfg, 21, {capi.OPT_STREAM_TRANSPORT: 0, capi.OPT_CLUSTER_TRANSPORT: 0})
    for x, y in zip(a, b):
        assert rel_err(x, y) < 1e-6


@pytest.mark.parametrize("n", [40, 48, 80])
def test_cluster_transport_matches_tiled_kernel(n):
    """Large planes: the cluster kernel (2 or 4 CTAs per plane) against the
    tiled kernel (27 x 27 tiles with recomputed halos) and the line walks."""
    cfg = small_cfg(ny=n, nz=n, nmu=4, nom=4, ng=2, ly=16.0, lz=16.0)
    ctx, _ = build(cfg, precision=capi.PREC_MIXED)
    a = _transport_states(ctx, cfg, 22, {capi.OPT_STREAM_TRANSPORT: 0, capi.OPT_CLUSTER_TRANSPORT: 1})
    b = _transport_states(ctx, cfg, 22, {capi.OPT_STREAM_TRANSPORT: 0, capi.OPT_CLUSTER_TRANSPORT: 0})
    c = _transport_states(ctx, cfg, 22, {capi.OPT_STREAM_TRANSPORT: 0, capi.OPT_CLUSTER_TRANSPORT: 0,
                                         capi.OPT_PLANE_TRANSPORT: 0})
    for x, y, z in zip(a, b, c):
        assert rel_err(x, y) < 1e-6
        assert rel_err(x, z) < 2e-6
    with pytest.raises(capi.BfpnError):
        ctx.set_option(capi.OPT_CLUSTER_TRANSPORT, 3)


def _edge_case_states(ctx, seed):
    """Seeded states with flat regions, differences below the limiter's
    epsilon and zero rows (as in the paired-angle test)."""
    Ng, nyz, NA = ctx.shape
    states = [a.reshape(Ng, nyz, NA).copy() for a in seeded_states(ctx, seed)]
    for a in states:
        a[1, : nyz // 2] = a[1, 0]
        a[min(2, Ng - 1)] = 3e-11 * np.arange(nyz)[:, None]
        a[0, ::7] = 0.0
    return [a.ravel() for a in states]


def _run_transports(ctx, cfg, states, opts):
    for k, v in opts.items():
        ctx.set_option(k, v)
    for k, arr in enumerate(states):
        ctx.set_state(k // 2, k % 2, arr)
    ctx.transport(0, 0, 0.5 * cfg.dt(), False)
    ctx.transport(0, 1, 0.5 * cfg.dt(), True)
    ctx.transport(1, 0, 0.31 * cfg.dt(), False)
    ctx.transport(1, 1, 0.5 * cfg.dt(), True)
    return [ctx.get_state(sp, cf) for sp in (0, 1) for cf in (0, 1)]


@pytest.mark.parametrize("n,nmu,nom", [(20, 6, 8), (16, 3, 4), (32, 5, 8)])
def test_stream_transport_matches_whole_plane_kernel(n, nmu, nom):
    """The row-streaming transport (z-stencil in registers, one row of the
    y-stencil in shared memory) against the whole-plane kernel, including flat
    regions, differences below the limiter's epsilon and partial 8-angle
    chunks (NA = 12, 40): the same operations in the same order per cell; the
    compiled kernels agree to one float rounding in a few per cent of cells
    (as the cluster kernel does), and the run is deterministic."""
    cfg = small_cfg(ny=n, nz=n, nmu=nmu, nom=nom, ng=5, lz=2.0)
    ctx, _ = build(cfg, precision=capi.PREC_MIXED)
    states = _edge_case_states(ctx, 31)
    a = _run_transports(ctx, cfg, states, {capi.OPT_STREAM_TRANSPORT: 2})
    a2 = _run_transports(ctx, cfg, states, {capi.OPT_STREAM_TRANSPORT: 2})
    b = _run_transports(ctx, cfg, states, {capi.OPT_STREAM_TRANSPORT: 0, capi.OPT_CLUSTER_TRANSPORT: 0})
    for x, x2, y in zip(a, a2, b):
        assert np.array_equal(x, x2)
        assert rel_err(x, y) < 1e-6
    assert np.abs(a[1]).max() > 0


@pytest.mark.parametrize("ny,nz", [(80, 80), (40, 33), (50, 127), (127, 3), (2, 45)])
def test_stream_transport_large_and_uneven_planes(ny, nz):
    """Planes without a whole-plane kernel, square or not, up to 128 wide:
    the row-streaming kernel against the line-walk kernel (float rounding),
    the tiled kernel and, on the same float-rounded state, the FP64 oracle."""
    cfg = small_cfg(ny=ny, nz=nz, nmu=3, nom=4, ng=2, ly=8.0, lz=6.0)
    ctx, ora = build(cfg, precision=capi.PREC_MIXED)
    states = [s.astype(np.float32).astype(np.float64) for s in _edge_case_states(ctx, 32)]
    a = _run_transports(ctx, cfg, states, {capi.OPT_STREAM_TRANSPORT: 1})
    b = _run_transports(ctx, cfg, states, {capi.OPT_STREAM_TRANSPORT: 0, capi.OPT_CLUSTER_TRANSPORT: 0,
                                           capi.OPT_PLANE_TRANSPORT: 0})
    for x, y in zip(a, b):
        assert rel_err(x, y) < 2e-6
    if ny >= 32 and nz >= 32:  # planes too large for one block also have the tiled kernel
        c = _run_transports(ctx, cfg, states, {capi.OPT_STREAM_TRANSPORT: 0, capi.OPT_CLUSTER_TRANSPORT: 0,
                                               capi.OPT_PLANE_TRANSPORT: 1})
        for x, z in zip(a, c):
            assert rel_err(x, z) < 2e-6
    set_both(ctx, ora, states)
    for (sp, cf, dtf, pres) in ((0, 0, 0.5, False), (0, 1, 0.5, True), (1, 0, 0.31, False), (1, 1, 0.5, True)):
        ora.transport(sp, cf, dtf * cfg.dt(), pres)
    for k, (sp, cf) in enumerate(((0, 0), (0, 1), (1, 0), (1, 1))):
        assert rel_err(a[k], ora.get_state(sp, cf)) < 2e-6
    with pytest.raises(capi.BfpnError):
        ctx.set_option(capi.OPT_STREAM_TRANSPORT, 3)


@pytest.mark.parametrize("flags", [{}, {"eq15_straggling": True, "trapezoidal_yz": True}])
def test_energy_ring_kernel_large_planes(flags):
    """Planes of at least 2^20 lanes (64 x 64 positions x 16 x 16 angles) take
    the mixed-precision energy sweep with a per-thread cp.async ring: the
    energy operator against the FP64 oracle on the same float-rounded state,
    and whole steps (fused IDD) against the FP64 path."""
    cfg = small_cfg(ny=63, nz=63, nmu=16, nom=16, ng=8, ly=8.0, lz=8.0, **flags)
    ctx, ora = build(cfg, precision=capi.PREC_MIXED)
    states = [a.astype(np.float32).astype(np.float64) for a in seeded_states(ctx, 31)]
    set_both(ctx, ora, states)
    ctx.energy(0, 0.5 * cfg.dt())
    ora.energy(0, 0.5 * cfg.dt())
    assert_states(ctx, ora, 1e-6, ((0, 0), (0, 1)))
    ctx.close()
    fp, _ = build(cfg)
    mix, _ = build(cfg, precision=capi.PREC_MIXED)
    i64, _ = fp.step(4)
    i32, _ = mix.step(4)
    assert rel_err(i32, i64) < 1e-5


def test_angle_operator():
    cfg = small_cfg(nmu=7, nom=6)
    ctx, ora = build(cfg)
    set_both(ctx, ora, seeded_states(ctx, 4))
    for sp, cf in ((0, 0), (1, 1)):
        ctx.angle(sp, cf, cfg.dt())
        ora.angle(sp, cf, cfg.dt())
    assert_states(ctx, ora, OP_TOL)


def test_idd_operator():
    cfg = small_cfg(trapezoidal_yz=True)
    ctx, ora = build(cfg)
    set_both(ctx, ora, seeded_states(ctx, 5))
    a, b = ctx.idd()
    c, d = ora.idd()
    assert abs(a - c) <= 1e-12 * abs(c)
    assert abs(b - d) <= 1e-12 * abs(d)


@pytest.mark.parametrize("flags", [
    {},
    {"trapezoidal_yz": True, "discrete_angle_delta": True, "normalize_initial_mass": True},
    {"no_spatial_clipping": True},
    {"primary_only": True},
    {"energy_only": True},
    {"no_transport": True},
    {"no_angle": True},
    {"legacy_energy": True},
    {"eq15_straggling": True},
    {"legacy_cross": True},
    {"material_name": "bone", "density": 1.85, "energy_density": 1.85},
])
def test_depth_steps_fp64(flags):
    flags = dict(flags)
    legacy_cross = flags.pop("legacy_cross", False)
    cfg = small_cfg(**flags)
    if legacy_cross:
        cfg.calibrate_cross_sections = True
    ctx, ora = build(cfg)
    n = 12
    idd_g, prox_g = ctx.step(n)
    idd_o, prox_o = ora.step(n)
    assert np.abs(idd_o).max() > 0
    assert rel_err(idd_g, idd_o) < STEP_TOL
    assert rel_err(prox_g, prox_o) < STEP_TOL
    assert_states(ctx, ora, STEP_TOL)


def test_depth_steps_tiled_transport():
    cfg = small_cfg(ny=40, nz=36, nmu=3, nom=2, ng=12, lg=20.0, beam_energy=15.0, ly=4.0, lz=4.0)
    ctx, ora = build(cfg)
    idd_g, _ = ctx.step(6)
    idd_o, _ = ora.step(6)
    assert rel_err(idd_g, idd_o) < STEP_TOL
    assert_states(ctx, ora, STEP_TOL)


def test_mixed_context_tables_equal_host_tables():
    """A float-state context keeps only the float angular kernel on the host;
    its table download still returns the double table, equal to the
    context-free builder's (and so to the oracle's)."""
    cfg = small_cfg(ny=8, nz=8, nmu=4, nom=4, ng=40, ly=2.0, lz=2.0)
    mu, sig = read_tables(table_dir("synthetic500"), cfg.ng)
    ctx, _ = build(cfg, precision=capi.PREC_MIXED)
    NA = cfg.nmu * cfg.nom
    for which, n in ((capi.TABLE_KER_V, cfg.ng * NA * NA), (capi.TABLE_KER_E1, cfg.ng ** 2)):
        assert np.array_equal(ctx.table(which, n), capi.host_table(cfg.grid(), cfg.phys(), mu, sig, which))


def _stepped(cfg, precision, overlap, calls, fused=0):
    ctx, ora = build(cfg, precision=precision)
    ctx.set_option(capi.OPT_STEP_OVERLAP, overlap)
    ctx.set_option(capi.OPT_FUSED_ENERGY, fused)
    idd = np.concatenate([ctx.step(n)[0] for n in calls])
    states = [ctx.get_state(sp, cf) for sp in (0, 1) for cf in (0, 1)]
    return ctx, ora, idd, states


@pytest.mark.parametrize("precision,overlap", [(capi.PREC_MIXED, 1), (capi.PREC_MIXED, 2), (capi.PREC_FP64, 2)])
def test_overlapped_steps_equal_sequential_steps(precision, overlap):
    """The secondary half of step n on a second stream beside the primary half
    of step n+1 (square planes: in-place transport), with (2) or without (1)
    the psi^2 T-A-T chains on streams of their own, gives the sequential
    order's IDD history and states bit for bit, over calls of 1, 2, 5 and 3
    steps (each call ends on whole steps)."""
    cfg = small_cfg(ny=8, nz=8, nmu=4, nom=4, ng=40, ly=2.0, lz=2.0)
    calls = [1, 2, 5, 3]
    _, _, idd_s, st_s = _stepped(cfg, precision, 0, calls)
    ctx, ora, idd_o, st_o = _stepped(cfg, precision, overlap, calls)
    assert np.abs(idd_s).max() > 0
    assert np.array_equal(idd_s, idd_o)
    for a, b in zip(st_s, st_o):
        assert np.array_equal(a, b)
    if precision == capi.PREC_FP64:
        idd_r, _ = ora.step(sum(calls))
        assert rel_err(idd_o, idd_r) < STEP_TOL
        assert_states(ctx, ora, STEP_TOL)


@pytest.mark.parametrize("straggling", [False, True])
def test_fused_energy_passes_equal_separate_passes(straggling):
    """The primary's closing energy pass of each step fused with the next
    step's opening pass (which also writes the source's operand) gives the
    separate passes' states bit for bit, over calls of 1, 2, 5 and 3 steps
    (each call opens its first step and closes its last); the IDD history
    agrees up to the order of the closing pass's partial sums (this plane is
    swept by the 2-lane register kernel when the passes are separate)."""
    cfg = small_cfg(ny=8, nz=8, nmu=4, nom=4, ng=40, ly=2.0, lz=2.0, eq15_straggling=straggling)
    calls = [1, 2, 5, 3]
    _, _, idd_s, st_s = _stepped(cfg, capi.PREC_MIXED, 0, calls)
    ctx, _, idd_f, st_f = _stepped(cfg, capi.PREC_MIXED, 2, calls, fused=1)
    assert ctx.kernels_per_step() > 0 and ctx.source_groups() > 0
    assert np.abs(idd_s).max() > 0
    assert np.abs(idd_f - idd_s).max() <= 1e-13 * np.abs(idd_s).max()
    for a, b in zip(st_s, st_f):
        assert np.array_equal(a, b)


def test_fused_energy_passes_tiny_values():
    """A 35 x 35 plane with 12 groups: a few psi^1 values about 1e-8 below
    the array's peak come out one float rounding step apart between the fused
    and the separate passes (4.6e-16 of the peak seen), so the states are
    compared to 1e-12 of their peak and bit for bit from 1e-6 of the peak up.
    The IDD agrees to the order of its partial sums."""
    cfg = small_cfg(nx=160, ny=34, nz=34, nmu=4, nom=4, ng=12, ly=8.0, lz=8.0, t_final=0.5)
    _, _, idd_s, st_s = _stepped(cfg, capi.PREC_MIXED, 0, [8])
    _, _, idd_f, st_f = _stepped(cfg, capi.PREC_MIXED, 2, [8], fused=1)
    assert np.abs(idd_f - idd_s).max() <= 1e-13 * np.abs(idd_s).max()
    for a, b in zip(st_s, st_f):
        peak = np.abs(a).max()
        assert np.abs(a - b).max() <= 1e-12 * peak
        big = np.abs(a) >= 1e-6 * peak
        assert np.array_equal(a[big], b[big])


def test_fused_energy_passes_large_plane_bit_identical():
    """On a plane of more than 2^20 lanes the separate passes use the 4-lane
    ring kernel, whose partial sums the fused kernel shares: the IDD history
    is bit-identical too."""
    cfg = small_cfg(ny=64, nz=64, nmu=16, nom=16, ng=24, ly=8.0, lz=8.0)
    calls = [3, 4]
    _, _, idd_s, st_s = _stepped(cfg, capi.PREC_MIXED, 0, calls)
    _, _, idd_f, st_f = _stepped(cfg, capi.PREC_MIXED, 2, calls, fused=1)
    assert np.abs(idd_s).max() > 0
    assert np.array_equal(idd_s, idd_f)
    for a, b in zip(st_s, st_f):
        assert np.array_equal(a, b)


def test_step_api_pieces_agree():
    """bfpn_step in one call == step by step == async + history download."""
    cfg = small_cfg()
    a, _ = build(cfg)
    b, _ = build(cfg)
    c, _ = build(cfg)
    ia, pa = a.step(9)
    ib = np.concatenate([b.step(1)[0] for _ in range(9)])
    c.step_async(4)
    c.step_async(5)
    c.sync()
    ic, pc = c.history()
    assert np.array_equal(ia, ib)
    assert np.array_equal(ia, ic) and np.array_equal(pa, pc)


@pytest.mark.parametrize("grid", ["8_7", "12_9"])
def test_reference_golden_full_run_fp64(grid):
    """All 1000 depth steps of the reference's golden water 230 MeV runs."""
    cfg = golden_config(grid)
    mu, sig = material_tables(cfg, "water")
    ctx = Context(cfg.grid(), cfg.phys(), capi.PREC_FP64)
    ctx.load_tables(mu, sig)
    ctx.init_beam()
    idd, _ = ctx.step(cfg.max_steps())
    gold = load_golden(grid)
    assert idd.shape[0] == gold.shape[0]
    assert rel_err(idd, gold[:, 1]) < STEP_TOL
    big = gold[:, 1] > 0.01 * gold[:, 1].max()
    assert (np.abs(idd - gold[:, 1])[big] / gold[big, 1]).max() < 1e-9


@pytest.mark.parametrize("flags", [{}, {"trapezoidal_yz": True, "discrete_angle_delta": True,
                                        "normalize_initial_mass": True}])
def test_lite_memory_steps_fp64(flags):
    """--lite-memory: psi^1 of the primary only, upwind energy step, lite IDD."""
    cfg = small_cfg(lite_memory=True, **flags)
    ctx, ora = build(cfg)
    n = 15
    idd_g, prox_g = ctx.step(n)
    idd_o, prox_o = ora.step(n)
    assert np.abs(idd_o).max() > 0 and not np.any(prox_o) and not np.any(prox_g)
    assert rel_err(idd_g, idd_o) < STEP_TOL
    assert rel_err(ctx.get_state(0, 0), ora.get_state(0, 0)) < STEP_TOL
    a, b = ctx.idd()
    assert abs(a - idd_g[-1]) <= 1e-12 * abs(a) and b == 0.0
    # only psi^1 of the primary exists, and the operators of the full path are not available
    for call in (lambda: ctx.get_state(0, 1), lambda: ctx.get_state(1, 0), lambda: ctx.energy(0, 0.1),
                 lambda: ctx.transport(0, 0, 0.1, False), lambda: ctx.angle(0, 0, 0.1),
                 lambda: ctx.secondary_source(), lambda: ctx.energy_moments(), lambda: ctx.spot_plane()):
        with pytest.raises(capi.BfpnError):
            call()
    big = make_config(ny=20, nz=20, nmu=20, nom=20, ng=500)  # device footprint: one array instead of eight
    lite = make_config(ny=20, nz=20, nmu=20, nom=20, ng=500, lite_memory=True)
    assert capi.footprint_bytes(lite.grid(), lite.phys()) < capi.footprint_bytes(big.grid(), big.phys()) / 7


def test_lite_memory_mixed_within_tolerance():
    cfg = small_cfg(lite_memory=True, t_final=8.0)
    mu, sig = read_tables(table_dir("synthetic500"), cfg.ng)
    out = []
    for prec in (capi.PREC_FP64, capi.PREC_MIXED):
        ctx = Context(cfg.grid(), cfg.phys(), prec)
        ctx.load_tables(mu, sig)
        ctx.init_beam()
        out.append(ctx.step(cfg.max_steps())[0])
    assert rel_err(out[1], out[0]) < 1e-5


def test_errors_are_reported_not_fatal():
    cfg = small_cfg()
    ctx = Context(cfg.grid(), cfg.phys())
    with pytest.raises(capi.BfpnError):
        ctx.step(1)  # tables not loaded
    mu, sig = read_tables(table_dir("synthetic500"), cfg.ng)
    with pytest.raises(capi.BfpnError):
        ctx.load_tables(mu[: cfg.ng - 3], sig)  # too few scattering rows
    with pytest.raises(capi.BfpnError):
        ctx.load_tables(mu, sig[:-1])  # sigma rows != Ng
    ctx.load_tables(mu, sig)
    with pytest.raises(capi.BfpnError):
        ctx.step(1)  # beam not initialised
    ctx.init_beam()
    ctx.step(2)
    with pytest.raises(capi.BfpnError):
        ctx.transport(3, 0, 0.1, False)


@pytest.mark.parametrize("shape", [dict(nmu=20, nom=20, ny=4, nz=4),   # NA 400: two output tiles of 208
                                   dict(nmu=7, nom=7, ny=9, nz=8),     # NA 49, 90 positions: two position tiles
                                   dict(nmu=3, nom=5, ny=2, nz=3)])    # NA 15: one padded tile
def test_tensor_core_source_mixed(shape):
    """tcgen05 split-bf16 angular contraction (mixed precision) against the
    FP64 oracle and against the fp32 CUDA-core path."""
    cfg = small_cfg(**shape)
    mu, sig = read_tables(table_dir("synthetic500"), cfg.ng)
    ctx = Context(cfg.grid(), cfg.phys(), capi.PREC_MIXED)
    ctx.load_tables(mu, sig)
    ctx.init_beam()
    ora = O.Oracle(cfg.grid(), cfg.phys(), mu, sig)
    F, f, F1, f1 = seeded_states(ctx, 11)
    for k, arr in enumerate((F, f, F1, f1)):
        # the mixed state holds floats: give the oracle the same rounded values
        arr32 = arr.astype(np.float32).astype(np.float64)
        ctx.set_state(k // 2, k % 2, arr32)
        ora.set_state(k // 2, k % 2, arr32)
    s_ref = ora.source()
    ctx.secondary_source()
    s_tc = ctx.source()
    assert rel_err(s_tc, s_ref) < 2e-5
    ctx.set_option(capi.OPT_TENSOR_CORES, 0)
    ctx.secondary_source()
    s_simt = ctx.source()
    assert rel_err(s_simt, s_ref) < 2e-6


def test_tensor_core_source_sparse_kernel_blocks():
    """Water's angular scattering kernel on a 20x20 angular grid keeps ~2 %
    of its entries (the rest fall below the reference's 1e-3 cut): the
    tensor-core contraction multiplies only the k chunks and column ranges of
    each 16 x 208 kernel block that hold non-zero entries.  Against the fp32
    CUDA-core contraction, which multiplies everything."""
    cfg = small_cfg(ny=6, nz=6, nmu=20, nom=20, ng=120, lg=259.0, beam_energy=230.0, sigma_e=2.3, ly=2.0, lz=2.0,
                    lu=1.0, lv=1.0)
    mu, sig = read_tables(table_dir("water"), cfg.ng)
    ctx = Context(cfg.grid(), cfg.phys(), capi.PREC_MIXED)
    ctx.load_tables(mu, sig)
    ctx.init_beam()
    assert ctx.source_groups() > 0
    F, f, F1, f1 = seeded_states(ctx, 5)
    for k, arr in enumerate((F, f, F1, f1)):
        ctx.set_state(k // 2, k % 2, arr.astype(np.float32).astype(np.float64))
    ctx.secondary_source()
    s_tc = ctx.source()
    ctx.set_option(capi.OPT_TENSOR_CORES, 0)
    ctx.secondary_source()
    s_simt = ctx.source()
    assert np.abs(s_simt).max() > 0
    assert rel_err(s_tc, s_simt) < 2e-5


def test_fp64_100mev_configuration_full_run():
    """The 100 MeV FP64 configuration (16x16 yz, 8x8 angles, 200 groups over
    104 MeV, 10 cm) against the oracle's full-run fixture, 1e-10 relative."""
    import os
    from conftest import GOLDEN
    from bfpn_gpu_b200 import parse_args
    fx = os.path.join(GOLDEN, "idd_c1_oracle.txt")
    header = open(fx).readline()
    args = header.split("oracle FP64:")[1].strip().split()
    cfg = parse_args(args)
    ref = np.loadtxt(fx)
    mu, sig = read_tables(table_dir("synthetic200_lg104"), cfg.ng)
    ctx = Context(cfg.grid(), cfg.phys(), capi.PREC_FP64)
    ctx.load_tables(mu, sig)
    ctx.init_beam()
    idd, proxy = ctx.step(cfg.max_steps())
    assert idd.shape[0] == ref.shape[0] == 250
    assert np.abs(idd - ref[:, 1]).max() <= 1e-10 * np.abs(ref[:, 1]).max()
    assert np.abs(proxy - ref[:, 2]).max() <= 1e-10 * np.abs(ref[:, 2]).max()
