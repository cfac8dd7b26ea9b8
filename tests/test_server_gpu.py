"""Multi-beam serving (bfpn_server_*) and batching (bfpn_batch_run): every
served beam's history equals a direct single-context run of the same beam."""
import numpy as np
import pytest

from conftest import table_dir
from bfpn_gpu_b200 import Context, capi, make_config, read_tables

pytestmark = pytest.mark.gpu


def cfg_of(**kw):
    base = dict(nx=120, ny=6, nz=5, nmu=4, nom=5, ng=40, ly=2.0, lz=1.5, lu=1.0, lv=1.2, lg=59.0, beam_energy=40.0,
                sigma_e=2.0, sigma_yz=0.4, material_name="water", t_final=2.0)
    base.update(kw)
    return make_config(**base)


BEAMS = [
    (dict(), capi.PREC_FP64),
    (dict(ny=8, nz=8, nmu=7, nom=7, trapezoidal_yz=True), capi.PREC_FP64),
    (dict(lite_memory=True), capi.PREC_FP64),
    (dict(primary_only=True, beam_energy=30.0), capi.PREC_FP64),
    (dict(ny=8, nz=8, nmu=6, nom=6), capi.PREC_MIXED),
    (dict(eq15_straggling=True, ng=50), capi.PREC_MIXED),
]


def direct(cfg, prec, mu, sig, n):
    ctx = Context(cfg.grid(), cfg.phys(), prec)
    ctx.load_tables(mu, sig)
    ctx.init_beam()
    out = ctx.step(n)
    ctx.close()
    return out


def requests():
    out = []
    for kw, prec in BEAMS:
        cfg = cfg_of(**kw)
        mu, sig = read_tables(table_dir("synthetic500"), cfg.ng)
        n = cfg.max_steps()
        out.append((cfg, prec, mu, sig, n, capi.make_beam(cfg.grid(), cfg.phys(), mu, sig, n, prec)))
    return out


def test_served_beams_equal_direct_runs():
    reqs = requests()
    with capi.Server(devices=(0,), workers_per_device=3) as srv:
        tickets = [srv.submit(r[-1]) for r in reqs]
        assert all(srv.poll(t) in (0, 1) for t in tickets)
        for (cfg, prec, mu, sig, n, _), t in zip(reqs, tickets):
            idd, prox, info = srv.wait(t, n)
            assert info["steps"] == n and info["device"] == 0 and info["run_ms"] > 0
            d_idd, d_prox = direct(cfg, prec, mu, sig, n)
            assert np.array_equal(idd, d_idd) and np.array_equal(prox, d_prox)
            assert srv.poll(t) == -1  # collected


def test_context_reuse_between_same_shape_beams():
    """One worker, the same grid with different beams: the kept context is
    reloaded and gives what a fresh context gives."""
    cfg_a, cfg_b = cfg_of(beam_energy=40.0), cfg_of(beam_energy=35.0, sigma_e=1.5)
    mu, sig = read_tables(table_dir("synthetic500"), cfg_a.ng)
    n = cfg_a.max_steps()
    with capi.Server(workers_per_device=1) as srv:
        ts = [srv.submit(capi.make_beam(c.grid(), c.phys(), mu, sig, n)) for c in (cfg_a, cfg_b, cfg_a)]
        res = [srv.wait(t, n)[0] for t in ts]
    assert np.array_equal(res[0], direct(cfg_a, capi.PREC_FP64, mu, sig, n)[0])
    assert np.array_equal(res[1], direct(cfg_b, capi.PREC_FP64, mu, sig, n)[0])
    assert np.array_equal(res[0], res[2])


def test_wait_timeout_and_errors():
    cfg = cfg_of(nx=400, t_final=40.0)  # 400 steps
    mu, sig = read_tables(table_dir("synthetic500"), cfg.ng)
    n = cfg.max_steps()
    with capi.Server(workers_per_device=1) as srv:
        t = srv.submit(capi.make_beam(cfg.grid(), cfg.phys(), mu, sig, n))
        with pytest.raises(capi.BfpnError) as e:
            srv.wait(t, n, timeout=0.0)
        assert e.value.status == capi.TIMEOUT or srv.poll(t) == 1
        idd, _, _ = srv.wait(t, n)  # still collectable
        assert idd.shape == (n,)
        with pytest.raises(capi.BfpnError):
            srv.wait(t, n)  # already collected
        bad = capi.make_beam(cfg.grid(), cfg.phys(), mu, sig[:-1], 3)  # sigma rows != Ng
        tb = srv.submit(bad)
        with pytest.raises(capi.BfpnError, match="load_tables"):
            srv.wait(tb, 3)
        with pytest.raises(capi.BfpnError):
            srv.submit(capi.make_beam(cfg.grid(), cfg.phys(), mu, sig, 0))  # nsteps < 1


def test_batch_run_matches_direct_runs():
    reqs = requests()
    out = capi.batch_run([r[-1] for r in reqs], workers_per_device=2)
    for (cfg, prec, mu, sig, n, _), (idd, prox) in zip(reqs, out):
        d_idd, d_prox = direct(cfg, prec, mu, sig, n)
        assert np.array_equal(idd, d_idd) and np.array_equal(prox, d_prox)


def _alone_mixed(r):
    ctx = Context(r.cfg.grid(), r.cfg.phys(), capi.PREC_MIXED)
    ctx.load_tables(r.mu, r.sigma)
    ctx.init_beam()
    idd, _ = ctx.step(r.nsteps)
    ctx.close()
    return idd


def test_continuous_batching_solo_equals_mix():
    """Bundle-eligible requests of three shape classes, submitted while
    earlier ones run: every served IDD equals the beam run alone on a context
    and the beam served alone, within 1e-6 of its peak."""
    import time

    from bfpn_gpu_b200 import beams

    pool = [r for r in beams.uneven_beams(24, seed=5, ny_choices=(16, 24, 32), na_choices=(12, 16))][:7]
    for r in pool:
        r.nsteps = min(r.nsteps, 45)
        assert capi.bundle_accepts(r.beam())
    with capi.Server(workers_per_device=1) as srv:
        tickets = []
        for k, r in enumerate(pool):
            tickets.append(srv.submit(r.beam()))
            if k in (1, 4):
                time.sleep(0.05)  # later requests arrive while the first run
        mix = [srv.wait(t, r.nsteps) for t, r in zip(tickets, pool)]
    with capi.Server(workers_per_device=1) as srv:
        solo = srv.wait(srv.submit(pool[0].beam()), pool[0].nsteps)[0]
    for r, (idd, _, info) in zip(pool, mix):
        ref = _alone_mixed(r)
        assert info["steps"] == r.nsteps
        assert np.abs(idd - ref).max() <= 1e-6 * np.abs(ref).max()
    assert np.abs(solo - mix[0][0]).max() <= 1e-6 * np.abs(solo).max()


def test_batching_off_serves_bit_identical_results():
    from bfpn_gpu_b200 import beams

    r = beams.uneven_beams(4, seed=9, ny_choices=(16,), na_choices=(12,))[0]
    r.nsteps = min(r.nsteps, 20)
    with capi.Server(workers_per_device=1, batching=False) as srv:
        idd = srv.wait(srv.submit(r.beam()), r.nsteps)[0]
        with pytest.raises(capi.BfpnError):
            srv.set_batching(True)  # only before the first submit
    assert np.array_equal(idd, _alone_mixed(r))
