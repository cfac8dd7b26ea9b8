"""Out-of-core mode (BFPN_FLAG_STREAMING_FULL, the reference's --streaming-full):
the state in pinned host memory, each depth step streamed through the GPU in
lane chunks (energy sweeps, source) and group chunks (transport, angular
diffusion).  Every cell sees the in-core kernels' arithmetic, so the states
equal an in-core run bit for bit and the IDD agrees to the rounding of its
differently grouped partial sums."""
import dataclasses
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_err, table_dir
from bfpn_gpu_b200 import Context, capi, make_config, parse_args, read_tables

pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "bfpn_gpu_b200", "bin", "bfp_solver")


def cfg_of(**kw):
    base = dict(nx=160, ny=6, nz=5, nmu=4, nom=5, ng=40, ly=2.0, lz=1.5, lu=1.0, lv=1.2, lg=59.0, beam_energy=40.0,
                sigma_e=2.0, sigma_yz=0.4, material_name="water", t_final=2.0)
    base.update(kw)
    return make_config(**base)


def run(cfg, prec, n, chunks=None):
    mu, sig = read_tables(table_dir("synthetic500"), cfg.ng)
    ctx = Context(cfg.grid(), cfg.phys(), prec)
    # the streamed step runs the primary's energy half-steps as separate
    # passes: compare with the resident run of the same order
    ctx.set_option(capi.OPT_FUSED_ENERGY, 0)
    if chunks:
        ctx.set_option(capi.OPT_LANE_CHUNK, chunks[0])
        ctx.set_option(capi.OPT_ENERGY_CHUNK, chunks[1])
    ctx.load_tables(mu, sig)
    ctx.init_beam()
    idd, prox = ctx.step(n)
    states = [ctx.get_state(sp, cf) for sp in (0, 1) for cf in (0, 1)]
    ctx.close()
    return idd, prox, states


def compare(cfg, prec, n, chunks):
    idd0, prox0, st0 = run(cfg, prec, n)
    ocfg = dataclasses.replace(cfg, streaming_full=True)
    idd1, prox1, st1 = run(ocfg, prec, n, chunks)
    for a, b in zip(st1, st0):
        assert np.array_equal(a, b)
    assert rel_err(idd1, idd0) < 1e-12
    assert np.abs(prox1 - prox0).max() <= 1e-9 * np.abs(prox0).max()


@pytest.mark.parametrize("prec", [capi.PREC_FP64, capi.PREC_MIXED])
@pytest.mark.parametrize("flags", [{}, {"eq15_straggling": True, "trapezoidal_yz": True},
                                   {"legacy_energy": True}])
def test_out_of_core_steps_equal_in_core(prec, flags):
    """Lane chunks of 5 positions (100 lanes; 42 positions make 9 chunks, the
    last partial) and group chunks of 7 groups (the last partial) against the
    resident run."""
    compare(cfg_of(**flags), prec, 25, (5 * 20 + 3, 7))


@pytest.mark.parametrize("prec", [capi.PREC_FP64, capi.PREC_MIXED])
def test_out_of_core_one_chunk_each_way(prec):
    """Chunks larger than the grid: one lane chunk and one group chunk."""
    compare(cfg_of(), prec, 20, (10 ** 7, 1000))


@pytest.mark.parametrize("n,prec", [(34, capi.PREC_FP64), (34, capi.PREC_MIXED), (40, capi.PREC_MIXED)])
def test_out_of_core_large_planes(n, prec):
    """Planes without a whole-plane kernel: the tiled transport (out of place,
    through the device scratch chunk) and the cluster kernel (40 x 40)."""
    cfg = cfg_of(ny=n, nz=n, nmu=4, nom=4, ng=12, ly=8.0, lz=8.0, t_final=0.5)
    compare(cfg, prec, 8, (160 * 16, 5))  # 160-position lane chunks, the last partial


def test_out_of_core_rejects_resident_only_calls():
    cfg = cfg_of(streaming_full=True)
    mu, sig = read_tables(table_dir("synthetic500"), cfg.ng)
    ctx = Context(cfg.grid(), cfg.phys(), capi.PREC_FP64)
    ctx.load_tables(mu, sig)
    ctx.init_beam()
    ctx.step(2)
    for call in (lambda: ctx.energy(0, 0.1), lambda: ctx.transport(0, 0, 0.1, False), lambda: ctx.angle(0, 0, 0.1),
                 lambda: ctx.secondary_source(), lambda: ctx.idd(), lambda: ctx.energy_moments(),
                 lambda: ctx.spot_plane()):
        with pytest.raises(capi.BfpnError, match="out-of-core"):
            call()
    with pytest.raises(capi.BfpnError):
        ctx.set_option(capi.OPT_LANE_CHUNK, 0)
    ctx.close()


def test_cli_streaming_full_matches_resident_run(tmp_path):
    """bfp_solver --streaming-full: the IDD of the resident run at every
    --idd-stride-th step and the last, the proxy file written as zeros (the
    reference's streaming output)."""
    common = ("60 --time 6 --data %s --lg 59 --ng 40 --energy 40 --sigma-e 2 --sigma-yz 0.4 --ny 6 --nz 5 "
              "--nmu 4 --nom 5 --ly 2 --lz 1.5 --lu 1 --lv 1.2" % table_dir("synthetic500")).split()
    outs = {}
    for name, extra in (("res", []), ("ooc", ["--streaming-full", "--lane-chunk", "50", "--energy-chunk", "9",
                                             "--idd-stride", "4"])):
        d = tmp_path / name
        d.mkdir()
        r = subprocess.run([CLI] + common + extra, cwd=d, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr + r.stdout
        outs[name] = (np.loadtxt(d / "idd_output.txt", ndmin=2), np.loadtxt(d / "dose_output.txt", ndmin=2), r.stdout)
    res, ooc = outs["res"], outs["ooc"]
    assert "Mode: streaming-full out-of-core" in ooc[2]
    n = res[0].shape[0]
    keep = [i for i in range(n) if (i + 1) % 4 == 0 or i + 1 == n]
    assert ooc[0].shape[0] == len(keep)
    assert np.array_equal(ooc[0][:, 0], res[0][keep, 0])
    assert np.abs(ooc[0][:, 1] - res[0][keep, 1]).max() <= 1e-12 * np.abs(res[0][:, 1]).max()
    assert not np.any(ooc[1][:, 1])
