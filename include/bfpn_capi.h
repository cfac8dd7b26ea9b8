/*
 * bfpn_capi.h -- C ABI of the B200 BFPn pencil-beam depth-step solver.
 *
 * Plain C types only: pointers, sizes, doubles and ints.  No CUDA or torch
 * types appear in the signatures, so any FFI (ctypes, cgo, JNI) can bind it.
 *
 * Phase-space layout (HBM, one array per species x DG coefficient):
 *     index = (ek * nyz + pos) * NA + ang
 *     pos   = iz * (Ny + 1) + iy          nyz = (Ny + 1) * (Nz + 1)
 *     ang   = iv * Nom + iu               NA  = Nmu * Nom
 * which is the index order of the reference (bfpm_solver.cu:1996,
 * spatial_transport.cu:46-47).  species 0 = primary, 1 = secondary;
 * coef 0 = psi^1 (F), coef 1 = psi^2 (f).
 *
 * Every function returns a bfpn_status; on failure bfpn_last_error(ctx)
 * gives a message.  Nothing here calls exit().
 */
#ifndef BFPN_CAPI_H
#define BFPN_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum bfpn_status {
    BFPN_OK = 0,
    BFPN_INVALID_ARG = 1,
    BFPN_OOM = 2,
    BFPN_CUDA_ERROR = 3,
    BFPN_TIMEOUT = 4,
    BFPN_IO_ERROR = 5,
    BFPN_NOT_READY = 6,
    BFPN_NO_DEVICE = 7
} bfpn_status;

/* Grid sizes and domain widths.  Mirrors GridParams (bfpm_solver.cuh:21-27);
 * the deltas are derived as in GridParams::computeDeltas
 * (bfpm_solver.cu:1116-1127): dt=Lx/Nx, dy=Ly/Ny, dz=Lz/Nz, dg=Lg/Ng,
 * du=Lu/(Nom+1), dv=Lv/(Nmu+1). */
typedef struct bfpn_grid {
    int32_t Nx, Ny, Nz, Ng, Nmu, Nom;
    double Lx, Ly, Lz, Lu, Lv, Lg;
} bfpn_grid;

/* Material presets (main.cu:123-138); selects the Bethe composition used
 * by the stopping-power ratio (bfpm_solver.cu:184-196). */
enum {
    BFPN_MATERIAL_NONE = 0, /* no --material given: water composition */
    BFPN_MATERIAL_WATER = 1,
    BFPN_MATERIAL_BONE = 2,
    BFPN_MATERIAL_AIR = 3
};

/* Physics / mode switches (PhysicsParams, bfpm_solver.cuh:30-62). */
enum {
    BFPN_FLAG_PRIMARY_ONLY = 1u << 0,
    BFPN_FLAG_LEGACY_ENERGY = 1u << 1,
    BFPN_FLAG_EQ15_STRAGGLING = 1u << 2,
    BFPN_FLAG_SAVE_ENERGY_MOMENTS = 1u << 3,
    BFPN_FLAG_ENERGY_ONLY = 1u << 4,
    BFPN_FLAG_NO_TRANSPORT = 1u << 5,
    BFPN_FLAG_NO_ANGLE = 1u << 6,
    BFPN_FLAG_NO_SPATIAL_CLIPPING = 1u << 7,
    BFPN_FLAG_DISCRETE_ANGLE_DELTA = 1u << 8,
    BFPN_FLAG_NORMALIZE_INITIAL_MASS = 1u << 9,
    BFPN_FLAG_TRAPEZOIDAL_YZ = 1u << 10,
    BFPN_FLAG_DOSE_CATASTROPHIC_LOSS = 1u << 11,
    BFPN_FLAG_CALIBRATE_CROSS_SECTIONS = 1u << 12,
    BFPN_FLAG_LITE_MEMORY = 1u << 13,
    /* --streaming-full (solveStreamingFull, bfpm_solver.cu:3113-3236): the four
     * state arrays live in pinned host memory instead of HBM and each depth
     * step streams them through the GPU -- lane chunks (every group of a set of
     * whole positions) for the energy sweeps and the source, group chunks for
     * transport and angular diffusion; chunk sizes BFPN_OPT_LANE_CHUNK /
     * BFPN_OPT_ENERGY_CHUNK.  For grids whose state does not fit in HBM.  The
     * per-operator entry points, the one-off IDD, energy moments and spot
     * planes need a resident state and report BFPN_INVALID_ARG. */
    BFPN_FLAG_STREAMING_FULL = 1u << 14
};

typedef struct bfpn_phys {
    double sig_E;          /* initial energy Gaussian sigma, MeV */
    double a_1;            /* 1 / (2 sigma_yz^2) */
    double a_2;            /* 1 / (2 sigma_angle^2) */
    double C_c;            /* carried for interface parity; unused on the path */
    double beam_energy;    /* E0, MeV */
    double density;        /* g/cm^3; used by transport-angle factor and dose */
    double energy_density; /* density used inside the energy sweep */
    int32_t material;      /* BFPN_MATERIAL_* */
    uint32_t flags;        /* BFPN_FLAG_* */
} bfpn_phys;

/* Arithmetic of the device state.
 * FP64:  every operator in double (parity mode, 1e-10 relative to the oracle).
 * MIXED: float state; the energy DG/CN recursion, the source energy
 *        contraction accumulators and the IDD accumulation stay double. */
enum { BFPN_PREC_FP64 = 0, BFPN_PREC_MIXED = 1 };

/* Set-up tables that bfpn_table_download can return (sizes in doubles). */
enum {
    BFPN_TABLE_S_S = 0,      /* Ng+1 stopping power at the DG nodes */
    BFPN_TABLE_T_C = 1,      /* Ng straggling */
    BFPN_TABLE_SIG_TRG = 2,  /* Ng transport cross-section */
    BFPN_TABLE_SIGMA_C = 3,  /* Ng catastrophic cross-section as used */
    BFPN_TABLE_EN = 4,       /* Ng+1 energy nodes */
    BFPN_TABLE_OMEND = 5,    /* 2*NA directions (omega_y, omega_z) */
    BFPN_TABLE_KER_E1 = 6,   /* Ng*Ng */
    BFPN_TABLE_KER_E2 = 7,   /* Ng*Ng */
    BFPN_TABLE_KER_V = 8,    /* Ng*NA*NA, [src][in][out] */
    BFPN_TABLE_BAND = 9,     /* 2*Ng: begin, end source groups per output */
    BFPN_TABLE_BEAM_YZA = 10,/* nyz*NA transverse-angular beam factor */
    BFPN_TABLE_BEAM_E = 11   /* Ng energy beam factor */
};

typedef struct bfpn_ctx bfpn_ctx;

/* ---- version / errors ------------------------------------------------ */
const char* bfpn_version(void);
const char* bfpn_status_string(bfpn_status s);
/* Message of the last failure on ctx (or of the last failed bfpn_create when
 * ctx is NULL).  Valid until the next call on the same context. */
const char* bfpn_last_error(const bfpn_ctx* ctx);

/* ---- solver context: replaces BFPnSolver (bfpm_solver.cuh:97-253) ----- */

/* File part of BFPnSolver::initialize (bfpm_solver.cu:1435-1480): reads the
 * first Ng rows of <data_path>/data_cross.txt (data_b.txt / data_a.txt for a
 * bone / air directory) into mu (Ng*3, zero-filled) and of cross_total.txt
 * into sigma_c (Ng).  Returns BFPN_IO_ERROR when a file cannot be opened;
 * the row counts let the caller apply the reference's checks (done again by
 * bfpn_load_tables). */
bfpn_status bfpn_read_tables(const char* data_path, int32_t Ng, double* mu, int32_t* mu_rows,
                             double* sigma_c, int32_t* sigma_rows);


/* One set-up table (BFPN_TABLE_*) built on the host from the same inputs
 * bfpn_load_tables takes, without a context or a GPU.  *n_out receives the
 * table length; n = capacity of out in doubles. */
bfpn_status bfpn_host_table(const bfpn_grid* grid, const bfpn_phys* phys, const double* mu, int32_t mu_rows,
                            const double* sigma_c, int32_t sigma_rows, int32_t which, double* out, uint64_t n,
                            uint64_t* n_out);

/* Device bytes a context of this shape needs (state, source, work buffers,
 * tables; in mixed precision also the tensor-core source's operand buffers
 * at their largest).  Replaces the reference's preflightMemory estimate
 * (bfpm_solver.cu:1321-1433).  Pure host arithmetic; no GPU needed. */
bfpn_status bfpn_footprint_bytes(const bfpn_grid* grid, const bfpn_phys* phys,
                                 int precision, uint64_t* bytes);

/* BFPnSolver::BFPnSolver (bfpm_solver.cu:1171-1207) + allocateMemory.
 * device: CUDA ordinal.  Allocates all device memory up front. */
bfpn_status bfpn_create(const bfpn_grid* grid, const bfpn_phys* phys,
                        int precision, int device, bfpn_ctx** out);
bfpn_status bfpn_destroy(bfpn_ctx* ctx);

/* Table part of BFPnSolver::initialize (bfpm_solver.cu:1435-1568):
 * mu is mu_rows x 3 (mu1, mu2, mu3), sigma_c has sigma_rows values, both
 * as read from data_cross.txt / cross_total.txt.  Rows beyond mu_rows are
 * zero (the reference accepts Ng-1 rows); sigma_rows must equal Ng.
 * Builds S_s, T_c, sig_trg, ker_e1/e2, band limits, ker_v, directions and
 * the DST factors, and uploads them. */
bfpn_status bfpn_load_tables(bfpn_ctx* ctx, const double* mu, int32_t mu_rows,
                             const double* sigma_c, int32_t sigma_rows);

/* BFPnSolver::initializeDistribution, full mode (bfpm_solver.cu:1815-2026):
 * Gaussian y/z, near-delta angle, Gaussian energy; F = f1*f2, f = F1 = f1 = 0.
 * Also resets the step counter. */
bfpn_status bfpn_init_beam(bfpn_ctx* ctx);

/* nsteps depth steps of BFPnSolver::solve (bfpm_solver.cu:2166-2267):
 * stepPrimary, stepSecondary (skipped on the context's first step), IDD and
 * dose proxy.  idd_out / proxy_out (host, nsteps doubles each) may be NULL.
 * The steps run as one CUDA graph replay per step with no host sync inside;
 * the call returns after the last step completed. */
bfpn_status bfpn_step(bfpn_ctx* ctx, int32_t nsteps, double* idd_out, double* proxy_out);

/* Enqueue nsteps without waiting and without copying results back; results
 * stay in the device history (bfpn_history_download). */
bfpn_status bfpn_step_async(bfpn_ctx* ctx, int32_t nsteps);
bfpn_status bfpn_sync(bfpn_ctx* ctx);
/* Copy IDD / proxy history entries [first, first+count) to the host. */
bfpn_status bfpn_history_download(bfpn_ctx* ctx, int32_t first, int32_t count,
                                  double* idd_out, double* proxy_out);
int32_t bfpn_steps_done(const bfpn_ctx* ctx);

/* ---- per-operator entry points (the sub-solver calls of stepPrimary /
 *      stepSecondary, bfpm_solver.cu:3238-3394) -------------------------- */

/* EnergyDepositionSolver::solve (energy_solver.cu:444-506), in place on
 * (F, f) of `species`, half-step dt.  with_source=1 adds the secondary
 * source computed by bfpn_secondary_source (species 1 only), as
 * solveSecondaryFromPrimary does (energy_solver.cu:508-573). */
bfpn_status bfpn_energy_eq15(bfpn_ctx* ctx, int32_t species, double dt, int32_t with_source);

/* SpatialTransportSolver::solveEq18 (spatial_transport.cu:202-262) on one
 * array; preserve_sign=1 disables the max(.,0) clipping. */
bfpn_status bfpn_transport_eq18(bfpn_ctx* ctx, int32_t species, int32_t coef,
                                double dt, int32_t preserve_sign);

/* AngleDiffusionSolver::solveEq19 (angle_diffusion.cu:420-483) on one array
 * with step dt (the full depth step in the reference's use). */
bfpn_status bfpn_angle_eq19(bfpn_ctx* ctx, int32_t species, int32_t coef, double dt);

/* secondarySourceFromPrimaryKernel (energy_solver.cu:287-333): source of the
 * secondary species from the current primary state, into the context's
 * source buffer. */
bfpn_status bfpn_secondary_source(bfpn_ctx* ctx);

/* computeIntegratedDepthDose + computeScalarDoseProxy
 * (bfpm_solver.cu:3473-3502, 3418-3444) of the current state. */
bfpn_status bfpn_idd(bfpn_ctx* ctx, double* idd, double* proxy);

/* State transfer of one array (cells doubles, converted to the device
 * precision on upload). */
bfpn_status bfpn_state_upload(bfpn_ctx* ctx, int32_t species, int32_t coef, const double* host);
bfpn_status bfpn_state_download(bfpn_ctx* ctx, int32_t species, int32_t coef, double* host);
bfpn_status bfpn_source_download(bfpn_ctx* ctx, double* host);
uint64_t bfpn_cells(const bfpn_ctx* ctx);

/* One set-up table (BFPN_TABLE_*); n = capacity of host in doubles. */
bfpn_status bfpn_table_download(bfpn_ctx* ctx, int32_t which, double* host, uint64_t n);

/* Kernel classes of the per-kernel profile. */
enum {
    BFPN_KERNEL_ENERGY = 0,         /* energy sweep (with fused IDD partials) */
    BFPN_KERNEL_TRANSPORT = 1,      /* MUSCL predictor-corrector */
    BFPN_KERNEL_ANGLE = 2,          /* DST-I angular diffusion */
    BFPN_KERNEL_SOURCE_ANGULAR = 3, /* source: angular contraction */
    BFPN_KERNEL_SOURCE_ENERGY = 4,  /* source: banded energy contraction */
    BFPN_KERNEL_IDD = 5,            /* IDD partials / final sum */
    BFPN_KERNEL_ENERGY_FUSED = 6,   /* primary closing + next opening energy pass, source operand */
    BFPN_KERNEL_CLASSES = 7
};

/* With profiling on, steps run eagerly (no graph) and every launch is
 * bracketed by CUDA events on the context stream; bfpn_kernel_profile
 * returns, per kernel class, the summed device time (ms) and the launch count
 * since the last reset.  n = entries the arrays hold (BFPN_KERNEL_CLASSES). */
bfpn_status bfpn_set_profiling(bfpn_ctx* ctx, int32_t on);
bfpn_status bfpn_kernel_profile(bfpn_ctx* ctx, double* ms_out, int32_t* launches_out, int32_t n);
bfpn_status bfpn_kernel_profile_reset(bfpn_ctx* ctx);
/* Kernel launches one regular depth step issues (after the first step). */
int32_t bfpn_kernels_per_step(bfpn_ctx* ctx);
/* Source groups whose angular contraction the secondary source computes. */
int32_t bfpn_source_groups(bfpn_ctx* ctx);

/* Run-time options (take effect from the next step; graphs are re-captured).
 * BFPN_OPT_TENSOR_CORES: 1 (default) computes the source's angular and
 *   energy contractions on the tcgen05 tensor cores in mixed precision
 *   (split-bf16 operands, fp32 accumulation); 0 uses the fp32 CUDA-core
 *   kernels.
 * BFPN_OPT_CUDA_GRAPHS: 1 (default) replays each depth step as a CUDA graph.
 * BFPN_OPT_PLANE_TRANSPORT: 1 (default) runs the transport with the unrolled
 *   kernels: one block per whole plane for square planes with
 *   Ny = Nz in {4,6,8,10,12,14,16,20,24,32}, 27 x 27 tiles for planes too large
 *   for one block; 0 uses the general line-walk kernel; a larger value selects
 *   the angles per block (whole planes: 8 or 16 mixed, 4 or 8 FP64; tiles: 4 or
 *   8 mixed, 2 or 4 FP64).  All compute the same values.
 * BFPN_OPT_PAIRED_ANGLES: 1 (default) lets mixed-precision kernels carry
 *   two lines per thread on packed fp32x2 arithmetic: the whole-plane
 *   transport two angles (when NA is even and the angles of each pair
 *   (2i, 2i+1) share the signs of their direction cosines), the angular DST
 *   two rows / columns of a slice (even Nom = Nmu); 0 keeps one line per
 *   thread.  Same values.
 * BFPN_OPT_CLUSTER_TRANSPORT: 1 (default) runs the mixed-precision transport
 *   of square planes with Ny = Nz in {40,48,64,80,96,128} (paired angles) on
 *   thread-block clusters: 2 to 8 CTAs hold one plane in their shared memory
 *   and exchange edge rows through distributed shared memory, in place;
 *   2 also uses it for Ny = Nz = 20 (in place of the whole-plane kernel);
 *   0 leaves those planes to the tiled kernel.  Values agree with the other
 *   kernels to float rounding.
 * BFPN_OPT_LANE_CHUNK / BFPN_OPT_ENERGY_CHUNK (out-of-core mode only): lanes
 *   per lane chunk (rounded down to whole positions, at least one; default
 *   262,144, the reference's --lane-chunk) and groups per group chunk (default
 *   128, --energy-chunk); the device buffers are sized on the next step.
 * BFPN_OPT_STEP_OVERLAP: 2 (default) lets the secondary half of one depth
 *   step (source, secondary energy / transport / angular passes, the step's
 *   IDD) run on a second stream beside the primary half of the next step,
 *   inside one CUDA graph, and within each half runs the transport-angle-
 *   transport chain of psi^2 beside that of psi^1; 1 overlaps the halves
 *   only; 0 runs everything one kernel after the other.  Applies when graphs
 *   are on and the transport is in place (whole-plane or cluster kernels);
 *   every bfpn_step / bfpn_step_async call still ends on whole steps.  Same
 *   kernels on the same inputs: the same values.
 * BFPN_OPT_STREAM_TRANSPORT: 1 (default) runs the mixed-precision transport
 *   of planes without a whole-plane kernel (Ny + 1 <= 256, any Nz, paired
 *   angles) with the row-streaming kernel: one block per (group, 8-angle)
 *   plane walks the z rows, the z-stencil in registers and one row of the
 *   y-stencil in shared memory, in place; 2 also uses it where a whole-plane
 *   kernel exists; 0 leaves those planes to the cluster / tiled kernels.
 *   Same values as the whole-plane kernel.
 * BFPN_OPT_FUSED_ENERGY: 1 (default) runs, in mixed precision with step
 *   overlap on (eq15 energy, NA a multiple of 4, the tensor-core source), the
 *   primary's closing energy half-step of each step and the opening half-step
 *   of the next as one kernel, which also writes the source's split-bf16
 *   operand: per step one primary energy pass and the operand's pack pass
 *   fewer.  Within a bfpn_step call the secondary half of step n then runs
 *   beside the primary's transport and angular passes of step n+1; the call
 *   still ends on whole steps.  0 keeps the separate passes.  The states
 *   are the separate passes' bit for bit except a few values far below the
 *   peak, which may round one float step apart (within 1e-12 of the peak);
 *   the IDD agrees to the order of the closing pass's partial sums. */
enum {
    BFPN_OPT_TENSOR_CORES = 0,
    BFPN_OPT_CUDA_GRAPHS = 1,
    BFPN_OPT_PLANE_TRANSPORT = 2,
    BFPN_OPT_PAIRED_ANGLES = 3,
    BFPN_OPT_CLUSTER_TRANSPORT = 4,
    BFPN_OPT_LANE_CHUNK = 5,
    BFPN_OPT_ENERGY_CHUNK = 6,
    BFPN_OPT_STEP_OVERLAP = 7,
    BFPN_OPT_STREAM_TRANSPORT = 8,
    BFPN_OPT_FUSED_ENERGY = 9
};
bfpn_status bfpn_set_option(bfpn_ctx* ctx, int32_t option, int32_t value);

/* bfpn_step_async(nsteps) bracketed by CUDA events on the context stream;
 * waits and returns the device time of the steps in *elapsed_ms. */
bfpn_status bfpn_timed_steps(bfpn_ctx* ctx, int32_t nsteps, double* elapsed_ms);

/* Set-up quantities the reference prints during initialize
 * (bfpm_solver.cu:1476-1500, 1536-1540, 1878-1880). */
typedef struct bfpn_setup_info {
    int32_t mu_rows;          /* explicit scattering rows read */
    int32_t beam_group;       /* group of the beam energy */
    double beam_group_energy; /* its midpoint, MeV */
    double sigma_fitted;      /* sigma_c of that group before calibration */
    double sigma_used;        /* after the optional legacy calibration */
    double omega_center_y, omega_center_z;
    double spatial_mass, angular_mass, energy_mass, initial_scale;
} bfpn_setup_info;
bfpn_status bfpn_setup_summary(bfpn_ctx* ctx, bfpn_setup_info* out);

/* Per-group integrals of psi^1 and psi^2 (primary + secondary) over y, z, u,
 * v of the current state (energyMomentKernel, bfpm_solver.cu:311-360), the
 * Eq. 25 diagnostic: out[2*g] = psi^1 integral, out[2*g+1] = psi^2 integral. */
bfpn_status bfpn_energy_moments(bfpn_ctx* ctx, double* out);

/* YZ dose plane of the current state (spotDosePlaneKernel,
 * bfpm_solver.cu:433-475): plane[iz*(Ny+1)+iy] = du dv * sum over groups and
 * angles of the Eq. 24 dose of primary + secondary / density.  nyz doubles. */
bfpn_status bfpn_spot_plane(bfpn_ctx* ctx, double* plane);

/* ---- multi-beam batching and serving ------------------------------------
 * The reference runs one beam per process (main.cu:344-348).  These calls
 * serve many independent beams from a thread-safe queue.  Requests a bundle
 * can hold are batched continuously (bfpn_server_set_batching); the others
 * are worked by threads that each own one context (stream + CUDA graph) on
 * one device, so several beams run at once per GPU and across GPUs; such a
 * worker keeps its context between requests of the same shape and only
 * reloads tables and beam.  A worker-served beam's IDD / proxy history is the
 * one bfpn_step on a fresh context gives; a batched beam's equals it up to
 * the order of the IDD partial sums. */
typedef struct bfpn_beam {
    bfpn_grid grid;
    bfpn_phys phys;
    int32_t precision;       /* BFPN_PREC_* */
    int32_t nsteps;          /* depth steps to run (>= 1) */
    const double* mu;        /* mu_rows x 3, as for bfpn_load_tables (copied at submit) */
    int32_t mu_rows;
    const double* sigma_c;   /* sigma_rows values (copied at submit) */
    int32_t sigma_rows;
} bfpn_beam;

typedef struct bfpn_beam_info {
    int32_t steps;           /* steps run (0 on failure) */
    int32_t device;          /* device that ran it */
    double queue_ms;         /* submit -> start */
    double run_ms;           /* start -> finish (context set-up, tables, beam, steps) */
} bfpn_beam_info;

typedef struct bfpn_server bfpn_server;

/* Start workers_per_device threads on each listed device (NULL / 0 devices:
 * device 0). */
bfpn_status bfpn_server_create(const int32_t* devices, int32_t n_devices, int32_t workers_per_device,
                               bfpn_server** out);
/* Continuous batching (default on): requests a bundle can hold
 * (bfpn_bundle_accepts) are served by one scheduler thread per device that
 * admits them FIFO into bundles of their shape class, each admission checked
 * against free device memory by the beam's footprint, and advances all
 * bundles together in rounds of depth steps; beams join and leave between
 * rounds.  Off: every request goes to the context workers.  Call before the
 * first submit (BFPN_NOT_READY otherwise). */
bfpn_status bfpn_server_set_batching(bfpn_server* server, int32_t on);
/* Queue one beam; thread-safe.  *ticket identifies it for poll / wait. */
bfpn_status bfpn_server_submit(bfpn_server* server, const bfpn_beam* beam, uint64_t* ticket);
/* 1 finished (success or failure), 0 queued or running, -1 unknown ticket. */
int32_t bfpn_server_poll(bfpn_server* server, uint64_t ticket);
/* Wait (timeout_s < 0: no limit; BFPN_TIMEOUT when it runs out, the beam
 * stays collectable), then copy the histories (capacity >= nsteps; idd /
 * proxy may be NULL) and release the ticket.  Returns the beam's status. */
bfpn_status bfpn_server_wait(bfpn_server* server, uint64_t ticket, double timeout_s, double* idd, double* proxy,
                             int32_t capacity, bfpn_beam_info* info);
/* Finish queued and running beams, stop the workers, free the server. */
bfpn_status bfpn_server_destroy(bfpn_server* server);
/* Message of the last failed server / batch call on this thread. */
const char* bfpn_server_last_error(void);
/* Run n beams to completion on a temporary server; idd_out[i] / proxy_out[i]
 * hold beams[i].nsteps doubles (either array list may be NULL); status_out[i]
 * (may be NULL) receives each beam's status.  Returns the first failure. */
bfpn_status bfpn_batch_run(const bfpn_beam* beams, int32_t n, const int32_t* devices, int32_t n_devices,
                           int32_t workers_per_device, double* const* idd_out, double* const* proxy_out,
                           bfpn_status* status_out);

/* ---- bundles: beams of one shape class advanced together ---------------
 * No counterpart in the reference, which runs one beam per process
 * (main.cu:344-348).  A bundle holds up to max_slots mixed-precision beams
 * whose kernels share one shape class -- the same Ny+1 = Nz+1 plane, square
 * Nmu = Nom angular grid and energy model -- and advances all of them with
 * one launch per operator per depth step: the energy sweep, the transport
 * half-steps and the DST of both state arrays of every slot each run as a
 * single kernel over a device table of per-slot arguments; each slot's
 * secondary source runs on a parallel graph branch.  Slots keep their own Ng,
 * tables, beam, depth-step count and IDD history, and join or leave at any
 * step (continuous batching).  The step of the current slot set is one CUDA
 * graph.  Kernel variants (angles per transport block, DST ring stages,
 * energy kernel form) are timed per shape class on the bundle's first steps
 * and the fastest kept for the process (autotuning); all variants compute the
 * same states.  Each beam's IDD history equals its single-context run up to
 * the order of the IDD partial sums. */
typedef struct bfpn_bundle bfpn_bundle;

enum {
    BFPN_BUNDLE_OPT_AUTOTUNE = 1,          /* 1 (default) tune on first use, 0 use the defaults / settings below */
    BFPN_BUNDLE_OPT_TRANSPORT_ANGLES = 2,  /* 8 or 16 angles per whole-plane transport block (turns tuning off) */
    BFPN_BUNDLE_OPT_DST_STAGES = 3,        /* 2 or 3 DST ring stages (turns tuning off) */
    BFPN_BUNDLE_OPT_ENERGY_RING = 4        /* 1 ring energy kernel, 0 register kernel (turns tuning off) */
};

/* BFPN_OK when a bundle can hold the beam (host-side check of its precision,
 * flags and grid; bfpn_bundle_admit may still refuse it for memory), else
 * BFPN_INVALID_ARG with the reason in bfpn_bundle_last_error(NULL). */
bfpn_status bfpn_bundle_accepts(const bfpn_beam* beam);
bfpn_status bfpn_bundle_create(int32_t device, int32_t max_slots, bfpn_bundle** out);
bfpn_status bfpn_bundle_set_option(bfpn_bundle* bundle, int32_t option, int32_t value);
/* Admit one beam (precision must be BFPN_PREC_MIXED): checks its footprint
 * (bfpn_footprint_bytes) against the device's free memory less 512 MiB
 * (BFPN_OOM when it does not fit, nothing allocated), builds its context
 * (tables, initial beam) and gives it a free slot (*slot).  The first beam
 * fixes the shape class; a beam of another class gets BFPN_INVALID_ARG. */
bfpn_status bfpn_bundle_admit(bfpn_bundle* bundle, const bfpn_beam* beam, int32_t* slot);
/* Enqueue up to nsteps depth steps of every slot that has steps left (each
 * stops at its own nsteps) on the bundle's stream; returns without waiting. */
bfpn_status bfpn_bundle_step(bfpn_bundle* bundle, int32_t nsteps);
/* Wait for the enqueued steps; BFPN_TIMEOUT if a kernel's bounded wait ran out. */
bfpn_status bfpn_bundle_sync(bfpn_bundle* bundle);
/* Slots that still have steps to run. */
int32_t bfpn_bundle_running(const bfpn_bundle* bundle);
/* Steps enqueued so far and steps requested of a slot (-1 / 0 when empty). */
bfpn_status bfpn_bundle_slot(const bfpn_bundle* bundle, int32_t slot, int32_t* steps_done, int32_t* nsteps);
/* Copy a finished slot's IDD / proxy histories (capacity >= its nsteps; either
 * may be NULL), then free the slot and its device memory. */
bfpn_status bfpn_bundle_collect(bfpn_bundle* bundle, int32_t slot, double* idd, double* proxy, int32_t capacity);
/* The tuning choice of the bundle's shape class as one line of text; returns
 * its length, or -1. */
int32_t bfpn_bundle_tuning(const bfpn_bundle* bundle, char* buf, int32_t buf_len);
/* cudaStream_t of the bundle. */
void* bfpn_bundle_stream(bfpn_bundle* bundle);
bfpn_status bfpn_bundle_destroy(bfpn_bundle* bundle);
/* Message of the bundle's last failure (NULL: the last failure on this thread). */
const char* bfpn_bundle_last_error(const bfpn_bundle* bundle);

/* ---- integrated depth dose without device allocation -------------------
 * No counterpart in the reference: its IDD (computeIntegratedDepthDose +
 * computeScalarDoseProxy, bfpm_solver.cu:3473-3502, 3418-3444) always runs
 * inside a solver that owns its buffers.  This variant is for callers that may
 * not have a library allocate device memory -- a serving process that has
 * reserved the GPU for its own pool, or a framework whose caching allocator
 * owns the state and must stay the only allocator -- and for callers that
 * cannot take the device synchronisation cudaMalloc/cudaFree imply.  It
 * allocates nothing: the caller passes the state, the dose weights and the
 * output as device pointers, and the only working memory is a fixed 64 KiB
 * device array inside the library.
 *
 * Computes out[0] = IDD (both species) and out[1] = psi^2 proxy of the primary,
 * the two numbers bfpn_idd returns, from device arrays laid out as a context
 * holds them: [Ng][(Ny+1)(Nz+1)][Nmu*Nom], double for BFPN_PREC_FP64, float for
 * BFPN_PREC_MIXED.  F1/f1 (secondary) may both be NULL.  dose_coef is the
 * device array of 2*Ng doubles (weight of psi^1, weight of psi^2 per group:
 * (S mid + catastrophic term) dg / density and its psi^2 counterpart, as in
 * Eq. 24).  out is a device array of 2 doubles.  grid gives the sizes and
 * lengths; trapezoidal_yz halves the yz edge weights.  Work is enqueued on
 * `stream` (a cudaStream_t of `device`; NULL = legacy default stream) and the
 * call returns without waiting; the caller's current device is left as it was.
 *
 * Limits: (Ny+1)(Nz+1)*Nmu*Nom <= 4,194,304 lanes (the scratch holds 4096
 * block partials of 1024 lanes each); a larger plane returns
 * BFPN_INVALID_ARG with a message.  Every call looks up the scratch's device
 * address with the device current (so a cudaDeviceReset between calls is
 * safe); the first call on each device also loads the library's device code
 * there and should come before any stream capture on that device.  All calls on one device share the scratch:
 * calls that overlap in time on that device (two streams, two host threads)
 * race and give wrong results -- order them on one stream.  Errors are
 * reported through bfpn_last_error(NULL). */
bfpn_status bfpn_idd_noalloc(const bfpn_grid* grid, int32_t precision, int32_t trapezoidal_yz,
                             const void* F0, const void* f0, const void* F1, const void* f1,
                             const double* dose_coef, double* out, int32_t device, void* stream);

/* ---- devices (printGPUInfo, main.cu:25-42) ---------------------------- */
int32_t bfpn_device_count(void);
/* Free and total device memory of a device (cudaMemGetInfo with that device
 * current; the caller's current device is left as it was). */
bfpn_status bfpn_device_memory(int32_t device, uint64_t* free_bytes, uint64_t* total_bytes);
/* One line per device property in the reference's format; returns the number
 * of bytes written (excluding the terminating zero), or -1. */
int32_t bfpn_device_info(int32_t device, char* buf, int32_t buf_len);
/* Raw stream handle (cudaStream_t) of the context, for callers that order
 * their own work against it. */
void* bfpn_stream(bfpn_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* BFPN_CAPI_H */
