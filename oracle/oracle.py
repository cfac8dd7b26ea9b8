"""ctypes binding of oracle/liboracle.so -- test infrastructure only.

The oracle is the CPU FP64 restatement of the reference's eq15 depth step.
Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it, as
the checker; the product never imports this module.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


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


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so is not built (make -C oracle)")
        L = ctypes.CDLL(path)
        vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [ctypes.POINTER(Grid), ctypes.POINTER(Phys), dp, ctypes.c_int, dp,
                                    ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_max_threads.restype = ctypes.c_int
        L.oracle_use_direct_source.argtypes = [vp, ctypes.c_int]
        L.oracle_step.argtypes = [vp, ctypes.c_int, dp, dp]
        L.oracle_steps_done.argtypes = [vp]
        L.oracle_steps_done.restype = ctypes.c_int
        L.oracle_cells.argtypes = [vp]
        L.oracle_cells.restype = ctypes.c_ulonglong
        L.oracle_get_state.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
        L.oracle_set_state.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
        L.oracle_set_steps_done.argtypes = [vp, ctypes.c_int]
        L.oracle_energy.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.oracle_transport.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.oracle_angle.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.oracle_source.argtypes = [vp, dp]
        L.oracle_idd.argtypes = [vp, dp, dp]
        L.oracle_energy_moments.argtypes = [vp, dp]
        L.oracle_spot_plane.argtypes = [vp, dp]
        L.oracle_table.restype = ctypes.c_longlong
        L.oracle_table.argtypes = [vp, ctypes.c_int, dp, ctypes.c_ulonglong]
        L.oracle_read_tables.restype = ctypes.c_int
        L.oracle_read_tables.argtypes = [ctypes.c_char_p, ctypes.c_int, dp, ip, dp, ip]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def set_threads(n):
    lib().oracle_set_threads(int(n))


def max_threads():
    return int(lib().oracle_max_threads())


def read_tables(data_path, Ng):
    """Reference table loader semantics (bfpm_solver.cu:1435-1480)."""
    mu = np.zeros(Ng * 3)
    sig = np.zeros(Ng)
    r, s = ctypes.c_int(0), ctypes.c_int(0)
    rc = lib().oracle_read_tables(data_path.encode(), Ng, _dp(mu), ctypes.byref(r), _dp(sig), ctypes.byref(s))
    if rc != 0:
        raise FileNotFoundError("cannot open tables in " + data_path)
    return mu.reshape(Ng, 3)[: r.value].copy(), sig[: s.value].copy()


def _copy_struct(src, cls):
    out = cls()
    for name, _ in cls._fields_:
        setattr(out, name, getattr(src, name))
    return out


class Oracle:
    """One beam's FP64 state on the host, advanced by the restated operators."""

    def __init__(self, grid, phys, mu, sigma):
        L = lib()
        self.grid = _copy_struct(grid, Grid)
        self.phys = _copy_struct(phys, Phys)
        mu = np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
        sigma = np.ascontiguousarray(sigma, dtype=np.float64)
        err = ctypes.create_string_buffer(512)
        self._h = L.oracle_create(ctypes.byref(self.grid), ctypes.byref(self.phys), _dp(mu), len(mu) // 3,
                                  _dp(sigma), len(sigma), err, 512)
        if not self._h:
            raise ValueError("oracle: " + err.value.decode())
        self.cells = int(L.oracle_cells(self._h))

    def close(self):
        if self._h:
            lib().oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        g = self.grid
        return (g.Ng, (g.Ny + 1) * (g.Nz + 1), g.Nmu * g.Nom)

    def step(self, n=1):
        idd = np.zeros(n)
        proxy = np.zeros(n)
        lib().oracle_step(self._h, n, _dp(idd), _dp(proxy))
        return idd, proxy

    def steps_done(self):
        return int(lib().oracle_steps_done(self._h))

    def set_steps_done(self, n):
        lib().oracle_set_steps_done(self._h, int(n))

    def use_direct_source(self, on=True):
        lib().oracle_use_direct_source(self._h, 1 if on else 0)

    def get_state(self, species, coef):
        out = np.empty(self.cells)
        lib().oracle_get_state(self._h, species, coef, _dp(out))
        return out

    def set_state(self, species, coef, arr):
        arr = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        assert arr.size == self.cells
        lib().oracle_set_state(self._h, species, coef, _dp(arr))

    def energy(self, species, dt, with_source=False):
        lib().oracle_energy(self._h, species, dt, 1 if with_source else 0)

    def transport(self, species, coef, dt, preserve_sign):
        lib().oracle_transport(self._h, species, coef, dt, 1 if preserve_sign else 0)

    def angle(self, species, coef, dt):
        lib().oracle_angle(self._h, species, coef, dt)

    def source(self):
        out = np.empty(self.cells)
        lib().oracle_source(self._h, _dp(out))
        return out

    def idd(self):
        a, b = ctypes.c_double(0), ctypes.c_double(0)
        lib().oracle_idd(self._h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def energy_moments(self):
        out = np.empty(2 * self.grid.Ng)
        lib().oracle_energy_moments(self._h, _dp(out))
        return out

    def spot_plane(self):
        g = self.grid
        out = np.empty((g.Ny + 1) * (g.Nz + 1))
        lib().oracle_spot_plane(self._h, _dp(out))
        return out

    def table(self, which, n):
        out = np.empty(n)
        got = lib().oracle_table(self._h, which, _dp(out), n)
        if got < 0:
            raise ValueError("bad table id or size")
        return out[:got]
