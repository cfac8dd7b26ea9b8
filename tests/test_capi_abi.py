"""The C ABI library loads and exports every entry point include/bfpn_capi.h
declares; host-only entry points work without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden_config, material_tables, table_dir
from bfpn_gpu_b200 import capi, make_config, read_tables
from oracle import oracle as O

HEADER = os.path.join(ROOT, "include", "bfpn_capi.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bfpn_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert len(names) >= 30
    assert "bfpn_create" in names and "bfpn_step" in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(capi.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_every_symbol():
    missing = [n for n in declared_functions() if n not in capi.SIGNATURES]
    assert not missing, missing
    capi.lib()  # binds all signatures


def test_version_and_status_strings():
    assert b"sm_100a" in capi.lib().bfpn_version()
    assert capi.lib().bfpn_status_string(capi.OOM) == b"out of device memory"


def test_read_tables_matches_reference_loader_semantics():
    for name, ng in (("water", 500), ("bone", 500), ("air", 500), ("synthetic500", 200)):
        mu, sig = read_tables(table_dir(name), ng)
        mu_o, sig_o = O.read_tables(table_dir(name), ng)
        assert np.array_equal(mu, mu_o) and np.array_equal(sig, sig_o)
    mu, sig = read_tables(table_dir("water"), 500)
    assert mu.shape == (499, 3) and sig.shape == (500,)  # the water table omits its last row
    with pytest.raises(capi.BfpnError):
        read_tables(os.path.join(ROOT, "no_such_dir"), 10)


@pytest.mark.parametrize("case", ["golden", "bone", "synthetic", "calibrated", "gauss"])
def test_host_tables_bit_identical_to_oracle(case):
    if case == "golden":
        cfg = golden_config("8_7")
        tabs = "water"
    elif case == "bone":
        cfg = make_config(nx=1000, ny=4, nz=3, nmu=5, nom=6, ng=500, material_name="bone", density=1.85,
                          energy_density=1.85, sigma_yz=0.5, sigma_e=2.3)
        tabs = "bone"
    elif case == "calibrated":
        cfg = make_config(nx=400, ny=3, nz=3, nmu=4, nom=4, ng=500, calibrate_cross_sections=True, lu=2.0, lv=1.5)
        tabs = "water"
    elif case == "gauss":
        cfg = make_config(nx=400, ny=5, nz=4, nmu=4, nom=5, ng=200, lg=104.0, normalize_initial_mass=True,
                          trapezoidal_yz=True, beam_energy=100.0, sigma_yz=0.4)
        tabs = "synthetic200_lg104"
    else:
        cfg = make_config(nx=250, ny=6, nz=6, nmu=8, nom=8, ng=200, lg=104.0, ly=4.0, lz=4.0, beam_energy=100.0,
                          sigma_yz=0.4)
        tabs = "synthetic200_lg104"
    mu, sig = read_tables(table_dir(tabs), cfg.ng)
    ora = O.Oracle(cfg.grid(), cfg.phys(), mu, sig)
    NA, nyz = cfg.nmu * cfg.nom, (cfg.ny + 1) * (cfg.nz + 1)
    sizes = {capi.TABLE_S_S: cfg.ng + 1, capi.TABLE_T_C: cfg.ng, capi.TABLE_SIG_TRG: cfg.ng,
             capi.TABLE_SIGMA_C: cfg.ng, capi.TABLE_EN: cfg.ng + 1, capi.TABLE_OMEND: 2 * NA,
             capi.TABLE_KER_E1: cfg.ng ** 2, capi.TABLE_KER_E2: cfg.ng ** 2, capi.TABLE_KER_V: cfg.ng * NA * NA,
             capi.TABLE_BAND: 2 * cfg.ng, capi.TABLE_BEAM_YZA: nyz * NA, capi.TABLE_BEAM_E: cfg.ng}
    for which, n in sizes.items():
        ours = capi.host_table(cfg.grid(), cfg.phys(), mu, sig, which)
        ref = ora.table(which, n)
        assert ours.shape == ref.shape and np.array_equal(ours, ref), which


def test_host_table_rejects_bad_input():
    cfg = make_config(nx=100, ny=3, nz=3, nmu=3, nom=3, ng=50)
    mu, sig = read_tables(table_dir("synthetic500"), cfg.ng)
    with pytest.raises(capi.BfpnError):
        capi.host_table(cfg.grid(), cfg.phys(), mu[:40], sig, capi.TABLE_S_S)  # < Ng-1 rows
    with pytest.raises(capi.BfpnError):
        capi.host_table(cfg.grid(), cfg.phys(), mu, sig[:49], capi.TABLE_S_S)  # sigma rows != Ng
    with pytest.raises(capi.BfpnError):
        capi.host_table(cfg.grid(), cfg.phys(), mu, sig, 99)


def test_footprint_scales_with_grid_and_precision():
    c2 = make_config(ny=20, nz=20, nmu=20, nom=20, ng=500)
    b64 = capi.footprint_bytes(c2.grid(), c2.phys(), capi.PREC_FP64)
    b32 = capi.footprint_bytes(c2.grid(), c2.phys(), capi.PREC_MIXED)
    cells = c2.cells()
    assert 8 * cells * 8 <= b64 < 8 * cells * 8 * 1.5
    assert 0.5 < b32 / b64 < 0.8  # half the state bytes plus the tensor-core source's operand buffers
    bad = make_config(ny=0)
    with pytest.raises(capi.BfpnError):
        capi.footprint_bytes(bad.grid(), bad.phys())


def test_create_without_device_fails_cleanly():
    if capi.lib().bfpn_device_count() > 0:
        pytest.skip("a CUDA device is present")
    cfg = make_config(ny=2, nz=2, nmu=2, nom=2, ng=10)
    with pytest.raises(capi.BfpnError) as e:
        capi.Context(cfg.grid(), cfg.phys())
    assert e.value.status == capi.NO_DEVICE


def test_idd_noalloc_checks_arguments_before_any_device_work():
    # fake, never dereferenced addresses: every case fails validation first
    fake = 0x1000
    cfg = make_config(ny=4, nz=4, nmu=3, nom=3, ng=10)
    big = make_config(ny=127, nz=127, nmu=17, nom=17, ng=10)  # 128 * 128 * 289 lanes > 4096 * 1024
    with pytest.raises(capi.BfpnError, match="exceeds the 4194304 lanes") as e:
        capi.idd_noalloc(big.grid(), capi.PREC_FP64, False, fake, fake, None, None, fake, fake)
    assert e.value.status == capi.INVALID_ARG
    with pytest.raises(capi.BfpnError, match="both secondary arrays"):
        capi.idd_noalloc(cfg.grid(), capi.PREC_FP64, False, fake, fake, fake, None, fake, fake)
    with pytest.raises(capi.BfpnError, match="null"):
        capi.idd_noalloc(cfg.grid(), capi.PREC_MIXED, False, fake, fake, None, None, None, fake)
    with pytest.raises(capi.BfpnError, match="precision"):
        capi.idd_noalloc(cfg.grid(), 5, False, fake, fake, None, None, fake, fake)
    if capi.lib().bfpn_device_count() == 0:
        with pytest.raises(capi.BfpnError) as e:
            capi.idd_noalloc(cfg.grid(), capi.PREC_FP64, False, fake, fake, None, None, fake, fake)
        assert e.value.status == capi.NO_DEVICE


def test_server_without_device_fails_cleanly():
    if capi.lib().bfpn_device_count() > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(capi.BfpnError) as e:
        capi.Server()
    assert e.value.status == capi.NO_DEVICE
    cfg = make_config(ny=2, nz=2, nmu=2, nom=2, ng=10)
    mu, sig = read_tables(table_dir("synthetic500"), cfg.ng)
    with pytest.raises(capi.BfpnError):
        capi.batch_run([capi.make_beam(cfg.grid(), cfg.phys(), mu, sig, 2)])
    with pytest.raises(capi.BfpnError) as e:
        capi.Server(workers_per_device=0)
    assert e.value.status == capi.INVALID_ARG


def test_streaming_and_lite_memory_are_exclusive():
    from bfpn_gpu_b200 import make_config
    cfg = make_config(ny=4, nz=4, nmu=2, nom=2, ng=10, lite_memory=True)
    import dataclasses
    bad = dataclasses.replace(cfg, streaming_full=True)
    with pytest.raises(capi.BfpnError, match="mutually exclusive"):
        capi.Context(bad.grid(), bad.phys(), capi.PREC_FP64)


def test_bundle_without_device_fails_cleanly():
    """No GPU here: creating a bundle reports NO_DEVICE with a message."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(capi.BfpnError, match="no such device"):
        capi.Bundle(device=0, max_slots=4)
    with pytest.raises(capi.BfpnError, match="bad arguments"):
        capi.Bundle(device=0, max_slots=0)
