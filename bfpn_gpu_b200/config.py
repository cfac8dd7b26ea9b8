"""Run configuration with the reference command line's meaning.

`parse_args` restates the flag handling of the reference's main
(src/main.cu:44-356): the same flags, defaults and quirks (a later
--material resets the density set by --rho; the optional positional Nx;
Lx = 40 and Lg = 259 fixed unless --lg is given, an extension of this solver).
The native CLI (bfpn_gpu_b200/bin/bfp_solver) parses the same way in C++;
this module serves tests and benchmarks.
"""
import math
from dataclasses import dataclass, field

from . import capi

# include/config.hpp:21-35
DEFAULTS = dict(NX=4000, NY=10, NZ=10, NG=500, NMU=11, NOM=11, LX=40.0, LY=1.0, LZ=1.0, LU=1.0, LV=1.0, LG=259.0)
MATERIAL_DENSITY = {"water": 1.0, "bone": 1.757, "air": 0.001205}
MATERIAL_ID = {"": capi.MATERIAL_NONE, "water": capi.MATERIAL_WATER, "bone": capi.MATERIAL_BONE,
               "air": capi.MATERIAL_AIR}

_BOOL_FLAGS = {
    "--lite-memory": "lite_memory", "--streaming-full": "streaming_full", "--primary-only": "primary_only",
    "--eq15-straggling": "eq15_straggling", "--save-energy-moments": "save_energy_moments",
    "--energy-only": "energy_only", "--no-transport": "no_transport", "--no-angle": "no_angle",
    "--no-spatial-clipping": "no_spatial_clipping", "--no-zero-chunk-skip": "no_zero_chunk_skip",
    "--no-fused-stream-boundary": "no_fused_stream_boundary", "--profile-steps": "profile_steps",
    "--discrete-angle-delta": "discrete_angle_delta", "--normalize-initial-mass": "normalize_initial_mass",
    "--trapezoidal-yz": "trapezoidal_yz", "--test": "test_mode",
}


@dataclass
class RunConfig:
    data_path: str = "./data"
    data_path_set: bool = False
    material_name: str = ""
    t_final: float = 40.0
    nx: int = DEFAULTS["NX"]
    ny: int = DEFAULTS["NY"]
    nz: int = DEFAULTS["NZ"]
    ng: int = DEFAULTS["NG"]
    nmu: int = DEFAULTS["NMU"]
    nom: int = DEFAULTS["NOM"]
    ly: float = DEFAULTS["LY"]
    lz: float = DEFAULTS["LZ"]
    lu: float = DEFAULTS["LU"]
    lv: float = DEFAULTS["LV"]
    lg: float = DEFAULTS["LG"]
    beam_energy: float = 230.0
    sigma_e: float = 1.0
    sigma_yz: float = 0.1
    density: float = 1.0
    energy_density: float = 1.0
    lite_memory: bool = False
    streaming_full: bool = False
    lane_chunk: int = 262144
    energy_chunk: int = 128
    primary_only: bool = False
    legacy_energy: bool = False
    eq15_straggling: bool = False
    save_energy_moments: bool = False
    energy_only: bool = False
    no_transport: bool = False
    no_angle: bool = False
    no_spatial_clipping: bool = False
    no_zero_chunk_skip: bool = False
    no_fused_stream_boundary: bool = False
    profile_steps: bool = False
    discrete_angle_delta: bool = False
    normalize_initial_mass: bool = False
    trapezoidal_yz: bool = False
    dose_catastrophic_loss: bool = True
    calibrate_cross_sections: bool = False
    test_mode: bool = False
    idd_stride: int = 1
    spot_depths: list = field(default_factory=list)
    spot_prefix: str = "spot"
    precision: int = capi.PREC_FP64

    # -- derived -------------------------------------------------------------
    def grid(self):
        return capi.Grid(Nx=self.nx, Ny=self.ny, Nz=self.nz, Ng=self.ng, Nmu=self.nmu, Nom=self.nom,
                         Lx=DEFAULTS["LX"], Ly=self.ly, Lz=self.lz, Lu=self.lu, Lv=self.lv, Lg=self.lg)

    def flags(self):
        f = 0
        for cond, bit in ((self.primary_only, capi.FLAG_PRIMARY_ONLY), (self.legacy_energy, capi.FLAG_LEGACY_ENERGY),
                          (self.eq15_straggling, capi.FLAG_EQ15_STRAGGLING),
                          (self.save_energy_moments, capi.FLAG_SAVE_ENERGY_MOMENTS),
                          (self.energy_only, capi.FLAG_ENERGY_ONLY), (self.no_transport, capi.FLAG_NO_TRANSPORT),
                          (self.no_angle, capi.FLAG_NO_ANGLE),
                          (self.no_spatial_clipping, capi.FLAG_NO_SPATIAL_CLIPPING),
                          (self.discrete_angle_delta, capi.FLAG_DISCRETE_ANGLE_DELTA),
                          (self.normalize_initial_mass, capi.FLAG_NORMALIZE_INITIAL_MASS),
                          (self.trapezoidal_yz, capi.FLAG_TRAPEZOIDAL_YZ),
                          (self.dose_catastrophic_loss, capi.FLAG_DOSE_CATASTROPHIC_LOSS),
                          (self.calibrate_cross_sections, capi.FLAG_CALIBRATE_CROSS_SECTIONS),
                          (self.lite_memory, capi.FLAG_LITE_MEMORY),
                          (self.streaming_full, capi.FLAG_STREAMING_FULL)):
            if cond:
                f |= bit
        return f

    def phys(self):
        # main.cu:292-299: a_1 = 1/(2 sigma_yz^2), a_2 = 1/(2 (1e-6)^2)
        return capi.Phys(sig_E=self.sigma_e, a_1=1.0 / 2.0 / self.sigma_yz / self.sigma_yz,
                         a_2=1.0 / 2.0 / 1e-6 / 1e-6, C_c=1.0 / math.sqrt(2.0 * math.pi * 0.1 * 1e-6),
                         beam_energy=self.beam_energy, density=self.density, energy_density=self.energy_density,
                         material=MATERIAL_ID.get(self.material_name, capi.MATERIAL_NONE), flags=self.flags())

    def dt(self):
        return DEFAULTS["LX"] / self.nx

    def max_steps(self):
        # bfpm_solver.cu:2178
        return int(math.ceil(self.t_final / self.dt() - 1e-12))

    def resolved_data_path(self):
        # main.cu:257-259
        if not self.data_path_set and self.material_name:
            return "BFPn_CPU_Solver/" + self.material_name
        return self.data_path

    def cells(self):
        return (self.ny + 1) * (self.nz + 1) * self.nmu * self.nom * self.ng


class ArgError(ValueError):
    pass


def parse_args(argv):
    """Parse reference-style arguments (without the program name)."""
    c = RunConfig()
    i = 0
    n = len(argv)

    def nxt():
        nonlocal i
        i += 1
        return argv[i]

    while i < n:
        a = argv[i]
        has = i + 1 < n
        if a == "--data" and has:
            c.data_path = nxt()
            c.data_path_set = True
        elif a == "--time" and has:
            c.t_final = float(nxt())
        elif a == "--energy" and has:
            c.beam_energy = float(nxt())
        elif a == "--sigma-e" and has:
            c.sigma_e = float(nxt())
        elif a == "--rho" and has:
            c.density = float(nxt())
            c.energy_density = c.density
        elif a == "--ny" and has:
            c.ny = int(nxt())
        elif a == "--nz" and has:
            c.nz = int(nxt())
        elif a == "--ly" and has:
            c.ly = float(nxt())
        elif a == "--lz" and has:
            c.lz = float(nxt())
        elif a == "--lu" and has:
            c.lu = float(nxt())
        elif a == "--lv" and has:
            c.lv = float(nxt())
        elif a == "--lg" and has:  # extension: energy-domain width (fixed 259 in the reference)
            c.lg = float(nxt())
        elif a == "--ng" and has:
            c.ng = int(nxt())
        elif a == "--nmu" and has:
            c.nmu = int(nxt())
        elif a == "--nom" and has:
            c.nom = int(nxt())
        elif a == "--material" and has:
            m = nxt()
            c.material_name = m
            if m not in MATERIAL_DENSITY:
                raise ArgError("Unknown material: " + m)
            c.density = MATERIAL_DENSITY[m]
            c.energy_density = c.density
        elif a == "--energy-model" and has:
            m = nxt()
            if m == "legacy":
                c.legacy_energy = True
            elif m == "eq15":
                c.legacy_energy = False
            else:
                raise ArgError("Unknown energy model: " + m)
        elif a == "--precision" and has:  # extension: fp64 | mixed
            m = nxt()
            if m not in ("fp64", "mixed"):
                raise ArgError("Unknown precision: " + m)
            c.precision = capi.PREC_FP64 if m == "fp64" else capi.PREC_MIXED
        elif a in _BOOL_FLAGS:
            setattr(c, _BOOL_FLAGS[a], True)
        elif a == "--dose-catastrophic-loss":
            c.dose_catastrophic_loss = True
        elif a == "--stopping-power-dose-only":
            c.dose_catastrophic_loss = False
        elif a == "--no-cross-section-calibration":
            c.calibrate_cross_sections = False
        elif a == "--legacy-cross-section-calibration":
            c.calibrate_cross_sections = True
        elif a == "--sigma-yz" and has:
            c.sigma_yz = float(nxt())
        elif a == "--lane-chunk" and has:
            c.lane_chunk = int(nxt())
        elif a == "--energy-chunk" and has:
            c.energy_chunk = int(nxt())
        elif a == "--stream-dir" and has:
            nxt()  # the reference's backing-file directory; the out-of-core state is in pinned host memory
        elif a == "--idd-stride" and has:
            c.idd_stride = max(1, int(nxt()))
        elif a == "--spot-depths" and has:
            c.spot_depths = [float(x) for x in nxt().split(",") if x]
        elif a == "--spot-prefix" and has:
            c.spot_prefix = nxt()
        elif a and a[0] != "-":
            c.nx = int(a)
        i += 1
    if c.lite_memory and c.streaming_full:
        raise ArgError("--lite-memory and --streaming-full are mutually exclusive")
    return c


def make_config(**kw):
    """RunConfig from keyword overrides (field names as in RunConfig)."""
    c = RunConfig()
    for k, v in kw.items():
        if not hasattr(c, k):
            raise AttributeError(k)
        setattr(c, k, v)
    return c
