"""ctypes binding of the solver's C ABI (include/bfpn_capi.h).

The shared library lib/libbfpn_b200.so is built in tree by
bfpn_gpu_b200/csrc/Makefile (or __graft_entry__.build()).  Loading fails loudly
when it is missing: there is no fallback implementation.
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libbfpn_b200.so")

# bfpn_status
OK, INVALID_ARG, OOM, CUDA_ERROR, TIMEOUT, IO_ERROR, NOT_READY, NO_DEVICE = range(8)
# precision
PREC_FP64, PREC_MIXED = 0, 1
# materials
MATERIAL_NONE, MATERIAL_WATER, MATERIAL_BONE, MATERIAL_AIR = 0, 1, 2, 3
# flags
FLAG_PRIMARY_ONLY = 1 << 0
FLAG_LEGACY_ENERGY = 1 << 1
FLAG_EQ15_STRAGGLING = 1 << 2
FLAG_SAVE_ENERGY_MOMENTS = 1 << 3
FLAG_ENERGY_ONLY = 1 << 4
FLAG_NO_TRANSPORT = 1 << 5
FLAG_NO_ANGLE = 1 << 6
FLAG_NO_SPATIAL_CLIPPING = 1 << 7
FLAG_DISCRETE_ANGLE_DELTA = 1 << 8
FLAG_NORMALIZE_INITIAL_MASS = 1 << 9
FLAG_TRAPEZOIDAL_YZ = 1 << 10
FLAG_DOSE_CATASTROPHIC_LOSS = 1 << 11
FLAG_CALIBRATE_CROSS_SECTIONS = 1 << 12
FLAG_LITE_MEMORY = 1 << 13
FLAG_STREAMING_FULL = 1 << 14
# run-time options
(OPT_TENSOR_CORES, OPT_CUDA_GRAPHS, OPT_PLANE_TRANSPORT, OPT_PAIRED_ANGLES, OPT_CLUSTER_TRANSPORT, OPT_LANE_CHUNK,
 OPT_ENERGY_CHUNK, OPT_STEP_OVERLAP, OPT_STREAM_TRANSPORT, OPT_FUSED_ENERGY) = range(10)
# kernel classes of the profile
KERNEL_CLASSES = ["energy", "transport", "angle", "source_angular", "source_energy", "idd", "energy_fused"]
# tables
(TABLE_S_S, TABLE_T_C, TABLE_SIG_TRG, TABLE_SIGMA_C, TABLE_EN, TABLE_OMEND, TABLE_KER_E1, TABLE_KER_E2,
 TABLE_KER_V, TABLE_BAND, TABLE_BEAM_YZA, TABLE_BEAM_E) = range(12)


class Grid(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int32), ("Ny", ctypes.c_int32), ("Nz", ctypes.c_int32),
                ("Ng", ctypes.c_int32), ("Nmu", ctypes.c_int32), ("Nom", ctypes.c_int32),
                ("Lx", ctypes.c_double), ("Ly", ctypes.c_double), ("Lz", ctypes.c_double),
                ("Lu", ctypes.c_double), ("Lv", ctypes.c_double), ("Lg", ctypes.c_double)]


class Phys(ctypes.Structure):
    _fields_ = [("sig_E", ctypes.c_double), ("a_1", ctypes.c_double), ("a_2", ctypes.c_double),
                ("C_c", ctypes.c_double), ("beam_energy", ctypes.c_double),
                ("density", ctypes.c_double), ("energy_density", ctypes.c_double),
                ("material", ctypes.c_int32), ("flags", ctypes.c_uint32)]


class Beam(ctypes.Structure):
    _fields_ = [("grid", Grid), ("phys", Phys), ("precision", ctypes.c_int32), ("nsteps", ctypes.c_int32),
                ("mu", ctypes.POINTER(ctypes.c_double)), ("mu_rows", ctypes.c_int32),
                ("sigma_c", ctypes.POINTER(ctypes.c_double)), ("sigma_rows", ctypes.c_int32)]


class BeamInfo(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int32), ("device", ctypes.c_int32), ("queue_ms", ctypes.c_double),
                ("run_ms", ctypes.c_double)]


# every entry point of include/bfpn_capi.h with its ctypes signature
_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_i32 = ctypes.c_int32
SIGNATURES = {
    "bfpn_version": (ctypes.c_char_p, []),
    "bfpn_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "bfpn_last_error": (ctypes.c_char_p, [_vp]),
    "bfpn_read_tables": (ctypes.c_int, [ctypes.c_char_p, _i32, _dp, ctypes.POINTER(_i32), _dp,
                                        ctypes.POINTER(_i32)]),
    "bfpn_host_table": (ctypes.c_int, [ctypes.POINTER(Grid), ctypes.POINTER(Phys), _dp, _i32, _dp, _i32, _i32, _dp,
                                       ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    "bfpn_footprint_bytes": (ctypes.c_int, [ctypes.POINTER(Grid), ctypes.POINTER(Phys), ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_uint64)]),
    "bfpn_create": (ctypes.c_int, [ctypes.POINTER(Grid), ctypes.POINTER(Phys), ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(_vp)]),
    "bfpn_destroy": (ctypes.c_int, [_vp]),
    "bfpn_load_tables": (ctypes.c_int, [_vp, _dp, _i32, _dp, _i32]),
    "bfpn_init_beam": (ctypes.c_int, [_vp]),
    "bfpn_step": (ctypes.c_int, [_vp, _i32, _dp, _dp]),
    "bfpn_step_async": (ctypes.c_int, [_vp, _i32]),
    "bfpn_sync": (ctypes.c_int, [_vp]),
    "bfpn_history_download": (ctypes.c_int, [_vp, _i32, _i32, _dp, _dp]),
    "bfpn_steps_done": (_i32, [_vp]),
    "bfpn_energy_eq15": (ctypes.c_int, [_vp, _i32, ctypes.c_double, _i32]),
    "bfpn_transport_eq18": (ctypes.c_int, [_vp, _i32, _i32, ctypes.c_double, _i32]),
    "bfpn_angle_eq19": (ctypes.c_int, [_vp, _i32, _i32, ctypes.c_double]),
    "bfpn_secondary_source": (ctypes.c_int, [_vp]),
    "bfpn_idd": (ctypes.c_int, [_vp, _dp, _dp]),
    "bfpn_state_upload": (ctypes.c_int, [_vp, _i32, _i32, _dp]),
    "bfpn_state_download": (ctypes.c_int, [_vp, _i32, _i32, _dp]),
    "bfpn_source_download": (ctypes.c_int, [_vp, _dp]),
    "bfpn_cells": (ctypes.c_uint64, [_vp]),
    "bfpn_table_download": (ctypes.c_int, [_vp, _i32, _dp, ctypes.c_uint64]),
    "bfpn_set_profiling": (ctypes.c_int, [_vp, _i32]),
    "bfpn_kernel_profile": (ctypes.c_int, [_vp, _dp, ctypes.POINTER(_i32), _i32]),
    "bfpn_kernel_profile_reset": (ctypes.c_int, [_vp]),
    "bfpn_kernels_per_step": (_i32, [_vp]),
    "bfpn_timed_steps": (ctypes.c_int, [_vp, _i32, _dp]),
    "bfpn_set_option": (ctypes.c_int, [_vp, _i32, _i32]),
    "bfpn_source_groups": (_i32, [_vp]),
    "bfpn_setup_summary": (ctypes.c_int, [_vp, _vp]),
    "bfpn_energy_moments": (ctypes.c_int, [_vp, _dp]),
    "bfpn_spot_plane": (ctypes.c_int, [_vp, _dp]),
    "bfpn_idd_noalloc": (ctypes.c_int, [ctypes.POINTER(Grid), _i32, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _vp]),
    "bfpn_server_create": (ctypes.c_int, [ctypes.POINTER(_i32), _i32, _i32, ctypes.POINTER(_vp)]),
    "bfpn_server_submit": (ctypes.c_int, [_vp, ctypes.POINTER(Beam), ctypes.POINTER(ctypes.c_uint64)]),
    "bfpn_server_poll": (_i32, [_vp, ctypes.c_uint64]),
    "bfpn_server_wait": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.c_double, _dp, _dp, _i32,
                                        ctypes.POINTER(BeamInfo)]),
    "bfpn_server_destroy": (ctypes.c_int, [_vp]),
    "bfpn_server_last_error": (ctypes.c_char_p, []),
    "bfpn_batch_run": (ctypes.c_int, [ctypes.POINTER(Beam), _i32, ctypes.POINTER(_i32), _i32, _i32,
                                      ctypes.POINTER(_dp), ctypes.POINTER(_dp), ctypes.POINTER(ctypes.c_int)]),
    "bfpn_bundle_accepts": (ctypes.c_int, [ctypes.POINTER(Beam)]),
    "bfpn_bundle_create": (ctypes.c_int, [_i32, _i32, ctypes.POINTER(_vp)]),
    "bfpn_server_set_batching": (ctypes.c_int, [_vp, _i32]),
    "bfpn_bundle_set_option": (ctypes.c_int, [_vp, _i32, _i32]),
    "bfpn_bundle_admit": (ctypes.c_int, [_vp, ctypes.POINTER(Beam), ctypes.POINTER(_i32)]),
    "bfpn_bundle_step": (ctypes.c_int, [_vp, _i32]),
    "bfpn_bundle_sync": (ctypes.c_int, [_vp]),
    "bfpn_bundle_running": (_i32, [_vp]),
    "bfpn_bundle_slot": (ctypes.c_int, [_vp, _i32, ctypes.POINTER(_i32), ctypes.POINTER(_i32)]),
    "bfpn_bundle_collect": (ctypes.c_int, [_vp, _i32, _dp, _dp, _i32]),
    "bfpn_bundle_tuning": (_i32, [_vp, ctypes.c_char_p, _i32]),
    "bfpn_bundle_stream": (_vp, [_vp]),
    "bfpn_bundle_destroy": (ctypes.c_int, [_vp]),
    "bfpn_bundle_last_error": (ctypes.c_char_p, [_vp]),
    "bfpn_device_count": (_i32, []),
    "bfpn_device_memory": (ctypes.c_int, [_i32, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "bfpn_device_info": (_i32, [_i32, ctypes.c_char_p, _i32]),
    "bfpn_stream": (_vp, [_vp]),
}

_lib = None


def lib():
    """Load lib/libbfpn_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("bfpn_gpu_b200: %s is missing; build it with `make -C bfpn_gpu_b200/csrc` "
                               "or __graft_entry__.build()" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class BfpnError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s: %s" % (lib().bfpn_status_string(status).decode(), message))
        self.status = status


def _ptr(a):
    return a.ctypes.data_as(_dp)


def read_tables(data_path, Ng):
    """(mu rows x 3, sigma_c) as the reference's loader reads them."""
    mu = np.zeros(Ng * 3)
    sig = np.zeros(Ng)
    r, s = _i32(0), _i32(0)
    rc = lib().bfpn_read_tables(str(data_path).encode(), Ng, _ptr(mu), ctypes.byref(r), _ptr(sig), ctypes.byref(s))
    if rc != OK:
        raise BfpnError(rc, lib().bfpn_last_error(None).decode())
    return mu.reshape(Ng, 3)[: r.value].copy(), sig[: s.value].copy()


def host_table(grid, phys, mu, sigma, which):
    """One set-up table built on the host (no GPU needed)."""
    mu = np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    sigma = np.ascontiguousarray(sigma, dtype=np.float64)
    n = ctypes.c_uint64(0)
    L = lib()
    rc = L.bfpn_host_table(ctypes.byref(grid), ctypes.byref(phys), _ptr(mu), len(mu) // 3, _ptr(sigma), len(sigma),
                           which, None, 0, ctypes.byref(n))
    if rc != OK and n.value == 0:
        raise BfpnError(rc, L.bfpn_last_error(None).decode())
    out = np.empty(max(int(n.value), 1))
    rc = L.bfpn_host_table(ctypes.byref(grid), ctypes.byref(phys), _ptr(mu), len(mu) // 3, _ptr(sigma), len(sigma),
                           which, _ptr(out), out.size, ctypes.byref(n))
    if rc != OK:
        raise BfpnError(rc, L.bfpn_last_error(None).decode())
    return out[: int(n.value)]


def footprint_bytes(grid, phys, precision=PREC_FP64):
    out = ctypes.c_uint64(0)
    rc = lib().bfpn_footprint_bytes(ctypes.byref(grid), ctypes.byref(phys), precision, ctypes.byref(out))
    if rc != OK:
        raise BfpnError(rc, lib().bfpn_last_error(None).decode())
    return int(out.value)


def _server_error(rc):
    return BfpnError(rc, lib().bfpn_server_last_error().decode())


def make_beam(grid, phys, mu, sigma, nsteps, precision=PREC_FP64):
    """A bfpn_beam request; the returned object keeps its table arrays alive."""
    mu = np.ascontiguousarray(mu, dtype=np.float64).reshape(-1, 3)
    sigma = np.ascontiguousarray(sigma, dtype=np.float64)
    b = Beam(grid=grid, phys=phys, precision=precision, nsteps=int(nsteps), mu=_ptr(mu), mu_rows=mu.shape[0],
             sigma_c=_ptr(sigma), sigma_rows=sigma.size)
    b._keep = (mu, sigma)
    return b


class Server:
    """bfpn_server_*: a queue of independent beams served by worker threads,
    each owning one context on one device."""

    def __init__(self, devices=(0,), workers_per_device=1, batching=True):
        devs = (_i32 * len(devices))(*devices)
        h = _vp()
        rc = lib().bfpn_server_create(devs, len(devices), workers_per_device, ctypes.byref(h))
        if rc != OK:
            raise _server_error(rc)
        self._h = h
        if not batching:
            self.set_batching(False)

    def set_batching(self, on):
        rc = lib().bfpn_server_set_batching(self._h, 1 if on else 0)
        if rc != OK:
            raise _server_error(rc)

    def submit(self, beam):
        t = ctypes.c_uint64(0)
        rc = lib().bfpn_server_submit(self._h, ctypes.byref(beam), ctypes.byref(t))
        if rc != OK:
            raise _server_error(rc)
        return t.value

    def poll(self, ticket):
        return lib().bfpn_server_poll(self._h, ticket)

    def wait(self, ticket, nsteps, timeout=-1.0):
        """(idd, proxy, info dict) of a finished beam."""
        idd, prox, info = np.empty(nsteps), np.empty(nsteps), BeamInfo()
        rc = lib().bfpn_server_wait(self._h, ticket, timeout, _ptr(idd), _ptr(prox), nsteps, ctypes.byref(info))
        if rc != OK:
            raise _server_error(rc)
        return idd, prox, {"steps": info.steps, "device": info.device, "queue_ms": info.queue_ms,
                           "run_ms": info.run_ms}

    def close(self):
        if getattr(self, "_h", None):
            lib().bfpn_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def bundle_accepts(beam):
    """True when a bundle can hold the beam (host-side check)."""
    return lib().bfpn_bundle_accepts(ctypes.byref(beam)) == OK


# bundle options
BUNDLE_OPT_AUTOTUNE, BUNDLE_OPT_TRANSPORT_ANGLES, BUNDLE_OPT_DST_STAGES, BUNDLE_OPT_ENERGY_RING = 1, 2, 3, 4


class Bundle:
    """bfpn_bundle_*: mixed-precision beams of one shape class advanced
    together, one launch per operator per depth step for every slot."""

    def __init__(self, device=0, max_slots=16):
        h = _vp()
        rc = lib().bfpn_bundle_create(device, max_slots, ctypes.byref(h))
        if rc != OK:
            raise BfpnError(rc, lib().bfpn_bundle_last_error(None).decode())
        self._h = h
        self._beams = {}

    def _check(self, rc):
        if rc != OK:
            raise BfpnError(rc, lib().bfpn_bundle_last_error(self._h).decode())

    def set_option(self, option, value):
        self._check(lib().bfpn_bundle_set_option(self._h, option, value))

    def admit(self, beam):
        """Slot of the admitted beam (a make_beam request)."""
        slot = _i32(-1)
        self._check(lib().bfpn_bundle_admit(self._h, ctypes.byref(beam), ctypes.byref(slot)))
        self._beams[slot.value] = beam
        return slot.value

    def step(self, n):
        self._check(lib().bfpn_bundle_step(self._h, int(n)))

    def sync(self):
        self._check(lib().bfpn_bundle_sync(self._h))

    def running(self):
        return int(lib().bfpn_bundle_running(self._h))

    def slot(self, k):
        done, total = _i32(0), _i32(0)
        self._check(lib().bfpn_bundle_slot(self._h, k, ctypes.byref(done), ctypes.byref(total)))
        return done.value, total.value

    def collect(self, k):
        """(idd, proxy) of a finished slot; frees the slot."""
        _, n = self.slot(k)
        idd, prox = np.empty(n), np.empty(n)
        self._check(lib().bfpn_bundle_collect(self._h, k, _ptr(idd), _ptr(prox), n))
        self._beams.pop(k, None)
        return idd, prox

    def tuning(self):
        buf = ctypes.create_string_buffer(512)
        lib().bfpn_bundle_tuning(self._h, buf, 512)
        return buf.value.decode()

    def close(self):
        if getattr(self, "_h", None):
            lib().bfpn_bundle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def batch_run(beams, devices=(0,), workers_per_device=2):
    """bfpn_batch_run: [(idd, proxy)] per beam, raising on the first failure."""
    n = len(beams)
    arr = (Beam * n)(*beams)
    idd = [np.empty(b.nsteps) for b in beams]
    prox = [np.empty(b.nsteps) for b in beams]
    ip = (_dp * n)(*[_ptr(a) for a in idd])
    pp = (_dp * n)(*[_ptr(a) for a in prox])
    st = (ctypes.c_int * n)()
    devs = (_i32 * len(devices))(*devices)
    rc = lib().bfpn_batch_run(arr, n, devs, len(devices), workers_per_device, ip, pp, st)
    if rc != OK:
        raise _server_error(rc)
    return list(zip(idd, prox))


def idd_noalloc(grid, precision, trapezoidal_yz, F0, f0, F1, f1, dose_coef, out, device=0, stream=None):
    """bfpn_idd_noalloc: IDD and psi^2 proxy of caller-owned device arrays,
    with no device allocation by the library.

    F0, f0, F1, f1, dose_coef and out are device addresses (ints; F1 and f1
    may be None); the result lands in out[0:2] on `stream` (a raw
    cudaStream_t address, None = legacy default stream) without a wait.
    """
    rc = lib().bfpn_idd_noalloc(ctypes.byref(grid), precision, 1 if trapezoidal_yz else 0, F0, f0, F1, f1,
                                dose_coef, out, device, stream)
    if rc != OK:
        raise BfpnError(rc, lib().bfpn_last_error(None).decode())


class Context:
    """One beam on one GPU, through the C ABI.

    Mirrors the reference's BFPnSolver (bfpm_solver.cuh:97-253): construct,
    load_tables (the table part of initialize), init_beam, step.
    """

    def __init__(self, grid, phys, precision=PREC_FP64, device=0):
        L = lib()
        self.grid = grid
        self.phys = phys
        self.precision = precision
        h = _vp()
        rc = L.bfpn_create(ctypes.byref(grid), ctypes.byref(phys), precision, device, ctypes.byref(h))
        if rc != OK:
            raise BfpnError(rc, L.bfpn_last_error(None).decode())
        self._h = h
        self.cells = int(L.bfpn_cells(h))

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib().bfpn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc != OK:
            raise BfpnError(rc, lib().bfpn_last_error(self._h).decode())

    @property
    def shape(self):
        g = self.grid
        return (g.Ng, (g.Ny + 1) * (g.Nz + 1), g.Nmu * g.Nom)

    # -- set-up ------------------------------------------------------------
    def load_tables(self, mu, sigma):
        mu = np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
        sigma = np.ascontiguousarray(sigma, dtype=np.float64)
        self._check(lib().bfpn_load_tables(self._h, _ptr(mu), len(mu) // 3, _ptr(sigma), len(sigma)))

    def init_beam(self):
        self._check(lib().bfpn_init_beam(self._h))

    # -- stepping ----------------------------------------------------------
    def step(self, n=1, fetch=True):
        if not fetch:
            self._check(lib().bfpn_step(self._h, n, None, None))
            return None
        idd = np.zeros(n)
        proxy = np.zeros(n)
        self._check(lib().bfpn_step(self._h, n, _ptr(idd), _ptr(proxy)))
        return idd, proxy

    def step_async(self, n=1):
        self._check(lib().bfpn_step_async(self._h, n))

    def sync(self):
        self._check(lib().bfpn_sync(self._h))

    def history(self, first=0, count=None):
        done = self.steps_done()
        if count is None:
            count = done - first
        idd = np.zeros(count)
        proxy = np.zeros(count)
        self._check(lib().bfpn_history_download(self._h, first, count, _ptr(idd), _ptr(proxy)))
        return idd, proxy

    def steps_done(self):
        return int(lib().bfpn_steps_done(self._h))

    # -- operators ---------------------------------------------------------
    def energy(self, species, dt, with_source=False):
        self._check(lib().bfpn_energy_eq15(self._h, species, dt, 1 if with_source else 0))

    def transport(self, species, coef, dt, preserve_sign):
        self._check(lib().bfpn_transport_eq18(self._h, species, coef, dt, 1 if preserve_sign else 0))

    def angle(self, species, coef, dt):
        self._check(lib().bfpn_angle_eq19(self._h, species, coef, dt))

    def secondary_source(self):
        self._check(lib().bfpn_secondary_source(self._h))

    def source(self):
        out = np.empty(self.cells)
        self._check(lib().bfpn_source_download(self._h, _ptr(out)))
        return out

    def idd(self):
        a, b = ctypes.c_double(0), ctypes.c_double(0)
        self._check(lib().bfpn_idd(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    # -- state -------------------------------------------------------------
    def get_state(self, species, coef):
        out = np.empty(self.cells)
        self._check(lib().bfpn_state_download(self._h, species, coef, _ptr(out)))
        return out

    def set_state(self, species, coef, arr):
        arr = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        if arr.size != self.cells:
            raise ValueError("state has %d cells, expected %d" % (arr.size, self.cells))
        self._check(lib().bfpn_state_upload(self._h, species, coef, _ptr(arr)))

    def table(self, which, n):
        out = np.empty(n)
        self._check(lib().bfpn_table_download(self._h, which, _ptr(out), n))
        return out

    def stream(self):
        return lib().bfpn_stream(self._h)

    # -- profiling -----------------------------------------------------------
    def set_profiling(self, on):
        self._check(lib().bfpn_set_profiling(self._h, 1 if on else 0))

    def kernel_profile(self, reset=False):
        """{class: (total ms, launches)} of profiled launches since the last reset."""
        n = len(KERNEL_CLASSES)
        ms = np.zeros(n)
        cnt = (_i32 * n)()
        self._check(lib().bfpn_kernel_profile(self._h, _ptr(ms), cnt, n))
        if reset:
            self._check(lib().bfpn_kernel_profile_reset(self._h))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(KERNEL_CLASSES)}

    def kernels_per_step(self):
        return int(lib().bfpn_kernels_per_step(self._h))

    def timed_steps(self, n):
        """n depth steps bracketed by CUDA events on the context stream; device ms."""
        ms = ctypes.c_double(0)
        self._check(lib().bfpn_timed_steps(self._h, n, ctypes.byref(ms)))
        return float(ms.value)

    def set_option(self, option, value):
        self._check(lib().bfpn_set_option(self._h, option, int(value)))

    def source_groups(self):
        return int(lib().bfpn_source_groups(self._h))

    def spot_plane(self):
        g = self.grid
        out = np.zeros((g.Ny + 1) * (g.Nz + 1))
        self._check(lib().bfpn_spot_plane(self._h, _ptr(out)))
        return out

    def energy_moments(self):
        out = np.zeros(2 * self.grid.Ng)
        self._check(lib().bfpn_energy_moments(self._h, _ptr(out)))
        return out
