// C-ABI implementation: one beam's solver context (replaces BFPnSolver,
// bfpm_solver.cuh:97-253, for the in-memory eq15 path).
//
// The context owns all device memory, allocated up front.  A depth step is
// enqueued as a fixed sequence of kernels on the context stream and captured
// once into a CUDA graph; the IDD of each step is reduced on the device into a
// history array, so a run of steps needs no host synchronisation.

#include "../../include/bfpn_capi.h"
#include "common.cuh"
#include "context.cuh"
#include "tables.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <type_traits>
#include <string>
#include <vector>

using namespace bfpn;

namespace {

thread_local std::string g_create_error;

}  // namespace

namespace {

bfpn_status fail(bfpn_ctx* c, bfpn_status s, const std::string& msg) {
    if (c) c->err = msg;
    else g_create_error = msg;
    return s;
}

#define CUDA_TRY(ctx, expr)                                                                      \
    do {                                                                                         \
        cudaError_t _e = (expr);                                                                 \
        if (_e != cudaSuccess)                                                                   \
            return fail(ctx, _e == cudaErrorMemoryAllocation ? BFPN_OOM : BFPN_CUDA_ERROR,       \
                        std::string(#expr) + ": " + cudaGetErrorString(_e));                     \
    } while (0)

bool valid_grid(const bfpn_grid& g, std::string& why) {
    if (g.Nx <= 0 || g.Ny <= 0 || g.Nz <= 0 || g.Ng < 2 || g.Nmu <= 0 || g.Nom <= 0) {
        why = "grid sizes must be positive (Ng >= 2)";
        return false;
    }
    if (!(g.Lx > 0) || !(g.Ly > 0) || !(g.Lz > 0) || !(g.Lu > 0) || !(g.Lv > 0) || !(g.Lg > 0)) {
        why = "domain widths must be positive";
        return false;
    }
    if (g.Nmu * g.Nom > 4096) {
        why = "Nmu*Nom above 4096 is not supported";
        return false;
    }
    const long long cells = static_cast<long long>(g.Ny + 1) * (g.Nz + 1) * g.Nmu * g.Nom * g.Ng;
    if (cells <= 0 || cells > (1LL << 40)) {
        why = "phase space too large";
        return false;
    }
    return true;
}

struct Layout {
    long long cells, per_e;
    size_t elem;
    int part_blocks;
    int hist_cap;
};

Layout layout_of(const bfpn_grid& g, int prec, int energy_block) {
    Layout L;
    L.per_e = static_cast<long long>(g.Ny + 1) * (g.Nz + 1) * g.Nmu * g.Nom;
    L.cells = L.per_e * g.Ng;
    L.elem = prec == BFPN_PREC_FP64 ? sizeof(double) : sizeof(float);
    L.part_blocks = std::max({energy_grid(L.per_e, energy_block), idd_partials_grid(L.per_e),
                              lite_energy_grid(L.per_e)});
    L.hist_cap = std::max(2 * g.Nx + 16, 4096);
    return L;
}

uint64_t footprint(const bfpn_grid& g, int prec, bool lite) {
    const Layout L = layout_of(g, prec, 128);
    const uint64_t arr = static_cast<uint64_t>(L.cells) * L.elem;
    const uint64_t NA = static_cast<uint64_t>(g.Nmu) * g.Nom;
    uint64_t b = 0;
    if (lite) {  // psi^1 of the primary and the small tables (bfpm_solver.cu:1338-1345)
        b += arr;
        b += 2 * static_cast<uint64_t>(g.Ng) * g.Ng * sizeof(double);  // e1, e2
        b += 2 * static_cast<uint64_t>(g.Ng) * NA * L.elem;            // angle factors
        b += static_cast<uint64_t>(L.per_e) * sizeof(double);          // beam factor
        b += 4 * static_cast<uint64_t>(L.part_blocks) * sizeof(double);
        b += 2 * static_cast<uint64_t>(L.hist_cap) * sizeof(double);
        b += 64ull * g.Ng * sizeof(double) + (1u << 20);
        return b;
    }
    b += 4 * arr;   // F, f, F1, f1
    b += arr;       // transport target
    b += arr;       // source
    b += prec == BFPN_PREC_MIXED ? std::max<uint64_t>(2 * arr, umma_q_bytes(L.per_e, g.Ng))
                                 : 2 * arr;  // angular contractions
    b += static_cast<uint64_t>(g.Ng) * NA * NA * L.elem;           // ker_v
    b += 2 * static_cast<uint64_t>(g.Ng) * g.Ng * sizeof(double);  // e1, e2
    b += 2 * static_cast<uint64_t>(g.Ng) * NA * L.elem;            // angle factors
    b += static_cast<uint64_t>(L.per_e) * sizeof(double);          // beam factor
    b += 4 * static_cast<uint64_t>(L.part_blocks) * sizeof(double);
    b += 2 * static_cast<uint64_t>(L.hist_cap) * sizeof(double);
    b += 64ull * g.Ng * sizeof(double) + (1u << 20);               // small tables
    if (prec == BFPN_PREC_MIXED) {
        // tensor-core source, at most every group a source group: the packed
        // split-bf16 A operand, the B tiles of the angular kernel and the
        // energy stage's coefficient tiles (an upper bound: 2 Ng x Ng bf16 pairs)
        const int ntiles = (static_cast<int>(NA) + 255) / 256;
        const int nt = ((static_cast<int>(NA) + ntiles - 1) / ntiles + 15) / 16 * 16;
        b += umma_pack_bytes(g.Ng, (g.Ny + 1) * (g.Nz + 1), static_cast<int>(NA), 16);
        b += umma_blob_bytes(g.Ng, static_cast<int>(NA), nt, 16);
        b += 8ull * g.Ng * g.Ng;
    }
    return b;
}

template <typename T>
T* as(void* p) {
    return static_cast<T*>(p);
}

// Wraps one kernel launch: counts it and, with profiling on, brackets it with
// CUDA events on the context stream (resolved by collect_profile).
template <typename F>
cudaError_t prof(bfpn_ctx* c, int cls, F&& launch) {
    c->launches++;
    if (!c->profiling) return launch();
    cudaEvent_t ev[2];
    for (auto& e : ev) {
        if (c->ev_pool.empty()) {
            cudaError_t r = cudaEventCreate(&e);
            if (r != cudaSuccess) return r;
        } else {
            e = c->ev_pool.back();
            c->ev_pool.pop_back();
        }
    }
    cudaError_t r = cudaEventRecord(ev[0], c->stream);
    if (r != cudaSuccess) return r;
    r = launch();
    if (r != cudaSuccess) return r;
    r = cudaEventRecord(ev[1], c->stream);
    c->pending.push_back({cls, ev[0], ev[1]});
    return r;
}

// Adds the elapsed times of finished profiled launches to the totals.
cudaError_t collect_profile(bfpn_ctx* c) {
    if (c->pending.empty()) return cudaSuccess;
    cudaError_t r = cudaStreamSynchronize(c->stream);
    if (r != cudaSuccess) return r;
    for (auto& p : c->pending) {
        float ms = 0.f;
        r = cudaEventElapsedTime(&ms, p.a, p.b);
        if (r != cudaSuccess) return r;
        c->prof_ms[p.cls] += ms;
        c->prof_n[p.cls] += 1;
        c->ev_pool.push_back(p.a);
        c->ev_pool.push_back(p.b);
    }
    c->pending.clear();
    return cudaSuccess;
}

bfpn_status dalloc(bfpn_ctx* c, void** out, size_t bytes) {
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        char msg[256];
        std::snprintf(msg, sizeof msg, "device allocation of %.3f GiB failed: %s", bytes / 1073741824.0,
                      cudaGetErrorString(e));
        return fail(c, BFPN_OOM, msg);
    }
    c->allocs.push_back({p, bytes});
    *out = p;
    return BFPN_OK;
}

// Frees one buffer from dalloc (no-op for nullptr) and sets the pointer to nullptr.
void dfree(bfpn_ctx* c, void*& p) {
    if (!p) return;
    for (size_t i = 0; i < c->allocs.size(); ++i)
        if (c->allocs[i].p == p) {
            cudaFree(p);
            c->allocs.erase(c->allocs.begin() + static_cast<long>(i));
            break;
        }
    p = nullptr;
}

// Step graphs capture buffer addresses and kernel choices: dropped whenever
// either changes.
void drop_graphs(bfpn_ctx* c) {
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    c->graph_exec = nullptr;
    c->graph_key = -1;
    for (auto& g : c->ovl_exec) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    for (auto& g : c->fus_exec) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

void free_all(bfpn_ctx* c) {
    for (auto& p : c->pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    c->pending.clear();
    for (auto e : c->ev_pool) cudaEventDestroy(e);
    c->ev_pool.clear();
    drop_graphs(c);
    for (cudaEvent_t* e : {&c->ev_fork, &c->ev_pread, &c->ev_join, &c->ev_ff[0], &c->ev_ff[1], &c->ev_fj[0], &c->ev_fj[1]})
        if (*e) {
            cudaEventDestroy(*e);
            *e = nullptr;
        }
    for (cudaStream_t* st : {&c->s_sec, &c->s_f[0], &c->s_f[1]})
        if (*st) {
            cudaStreamDestroy(*st);
            *st = nullptr;
        }
    for (auto& b : c->allocs) cudaFree(b.p);
    c->allocs.clear();
    for (void* p : c->host_allocs) cudaFreeHost(p);
    c->host_allocs.clear();
}

// Transport launch shape: a whole (Ny+1) x (Nz+1) plane per block when it
// fits (updates in place); otherwise square tiles written to ctx->tmp.
void choose_transport(bfpn_ctx* c) {
    const size_t sz = c->elem;
    const int Ny1 = c->Ny + 1, Nz1 = c->Nz + 1;
    const size_t budget = 72 * 1024;  // three blocks per SM at least
    // whole plane per block, the widest angle chunk (32..128 contiguous bytes) that fits
    for (int ac : {32, 16, 8, 4}) {
        if (ac * sz > 128) continue;
        if (ac * sz < 32 && c->NA >= 8) break;
        if (transport_smem(Ny1, Nz1, Ny1, Nz1, ac, sz) <= budget) {
            c->tr_ac = ac;
            c->tr_ty = Ny1;
            c->tr_tz = Nz1;
            c->tr_inplace = true;
            return;
        }
    }
    // square tiles with 32-byte angle chunks, balanced over the plane
    const int ac = std::max(1, static_cast<int>(32 / sz));
    int tmax = 4;
    for (int cand = 64; cand >= 4; --cand)
        if (transport_smem(Ny1, Nz1, cand, cand, ac, sz) <= budget) {
            tmax = cand;
            break;
        }
    const int ky = (Ny1 + tmax - 1) / tmax, kz = (Nz1 + tmax - 1) / tmax;
    c->tr_ac = ac;
    c->tr_ty = (Ny1 + ky - 1) / ky;
    c->tr_tz = (Nz1 + kz - 1) / kz;
    c->tr_inplace = (c->tr_ty >= Ny1 && c->tr_tz >= Nz1);
}

// The unrolled whole-plane kernel, where one is compiled for this plane
// size; it works in place whatever the line-walk kernel's shape.
void choose_plane_transport(bfpn_ctx* c) {
    // 16 float / 4 double angles per block: 64 / 32 contiguous bytes per position
    // (16 float angles measured 7% faster than 8 on a 21x21 plane)
    c->tr_plane_ac = c->elem == 4 ? 16 : 4;
    c->tr_plane_ok = transport_plane_supported(c->Ny, c->Nz) &&
                     transport_plane_smem(c->Ny + 1, c->tr_plane_ac, c->elem) <= 200 * 1024;
    c->tr_plane = c->tr_plane_ok;
    // planes the line-walk kernel would tile: the unrolled tiled kernel instead
    // (8 float / 4 double angles per block: 78 KB of shared memory, 2 blocks per SM)
    c->tr_tile_ac = c->elem == 4 ? 8 : 4;
    c->tr_tile_ok = !c->tr_plane_ok && !c->tr_inplace;
    c->tr_tile = c->tr_tile_ok;
    c->tr_cluster_ok = c->elem == 4 && transport_cluster_supported(c->Ny, c->Nz);
    c->tr_stream_ok = c->elem == 4 && transport_stream_supported(c->Ny, c->NA);
}

// The row-streaming kernel runs this context's transport (it needs paired angles).
bool stream_transport(const bfpn_ctx* c) {
    if (!c->tr_stream_ok || !c->tr_pairs || !c->tr_pairs_ok) return false;
    return c->tr_stream == 2 || (c->tr_stream == 1 && !c->tr_plane);
}

// The cluster kernel runs this context's transport (it needs paired angles).
bool cluster_transport(const bfpn_ctx* c) {
    if (stream_transport(c)) return false;
    if (!c->tr_cluster_ok || !c->tr_pairs || !c->tr_pairs_ok) return false;
    return c->tr_cluster == 2 || (c->tr_cluster == 1 && !c->tr_plane);
}

bool transport_in_place(const bfpn_ctx* c) {
    return c->tr_plane || c->tr_inplace || cluster_transport(c) || stream_transport(c);
}

template <typename T>
bfpn_status upload_as(bfpn_ctx* c, void* dst, const double* host, size_t n) {
    if (sizeof(T) == sizeof(double)) {
        CUDA_TRY(c, cudaMemcpyAsync(dst, host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        return BFPN_OK;
    }
    // converted on the host's threads into a buffer they touch first
    std::unique_ptr<T[]> tmp(new T[n]);
    parallel_ranges(n, size_t(1) << 20, [&](size_t b, size_t e) {
        for (size_t i = b; i < e; ++i) tmp[i] = static_cast<T>(host[i]);
    });
    CUDA_TRY(c, cudaMemcpyAsync(dst, tmp.get(), n * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return BFPN_OK;
}

bfpn_status upload_state_table(bfpn_ctx* c, void* dst, const double* h, size_t n) {
    return c->prec == BFPN_PREC_FP64 ? upload_as<double>(c, dst, h, n) : upload_as<float>(c, dst, h, n);
}

template <typename V>
bfpn_status upload_state_table(bfpn_ctx* c, void* dst, const V& h) {
    return upload_state_table(c, dst, h.data(), h.size());
}

bfpn_status upload_f64(bfpn_ctx* c, void* dst, const void* host, size_t bytes) {
    CUDA_TRY(c, cudaMemcpyAsync(dst, host, bytes, cudaMemcpyHostToDevice, c->stream));
    return BFPN_OK;
}

// ---- operator enqueues (typed) ---------------------------------------------

template <typename T>
cudaError_t enq_energy(bfpn_ctx* c, int species, const double* coef, bool with_source, double* partials) {
    EnergyArgs<T> a;
    a.F = as<T>(c->st[species][0]);
    a.f = as<T>(c->st[species][1]);
    a.src = with_source ? as<const T>(c->src) : nullptr;
    a.coef = coef;
    a.Ng = c->Ng;
    a.lanes = c->per_e;
    if (c->p.flags & BFPN_FLAG_LEGACY_ENERGY) a.mode = EMODE_LEGACY;
    else if (c->p.flags & BFPN_FLAG_EQ15_STRAGGLING) a.mode = EMODE_EQ15_STRAG;
    else a.mode = EMODE_EQ15;
    a.partials = partials;
    a.dose_coef = c->dose_coef;
    a.NA = c->NA;
    a.Ny = c->Ny;
    a.Nz = c->Nz;
    a.trapezoidal = (c->p.flags & BFPN_FLAG_TRAPEZOIDAL_YZ) ? 1 : 0;
    return prof(c, BFPN_KERNEL_ENERGY, [&] { return launch_energy<T>(a, c->energy_block, c->stream); });
}

// ng >= 0: the arrays hold ng groups (a chunk of the out-of-core mode).
template <typename T>
cudaError_t enq_transport(bfpn_ctx* c, const void* in, void* out, double dt, bool preserve_sign, int ng = -1) {
    TransportArgs<T> a;
    a.in = as<const T>(const_cast<void*>(in));
    a.out = as<T>(out);
    a.omega = as<const T>(c->omega);
    a.Ny = c->Ny;
    a.Nz = c->Nz;
    a.NA = c->NA;
    a.Ng = ng >= 0 ? ng : c->Ng;
    a.dt = static_cast<T>(dt);
    a.dy = static_cast<T>(c->d.dy);
    a.dz = static_cast<T>(c->d.dz);
    a.tile_y = c->tr_ty;
    a.tile_z = c->tr_tz;
    a.preserve_sign = preserve_sign ? 1 : 0;
    a.pairs = (c->elem == 4 && c->tr_pairs && c->tr_pairs_ok) ? 1 : 0;
    if constexpr (sizeof(T) == 4) {
        if (stream_transport(c))
            return prof(c, BFPN_KERNEL_TRANSPORT, [&] { return launch_transport_stream(a, c->stream); });
        if (cluster_transport(c))
            return prof(c, BFPN_KERNEL_TRANSPORT, [&] { return launch_transport_cluster(a, c->stream); });
    }
    if (c->tr_plane)
        return prof(c, BFPN_KERNEL_TRANSPORT, [&] { return launch_transport_plane<T>(a, c->tr_plane_ac, c->stream); });
    if (c->tr_tile && a.in != a.out)
        return prof(c, BFPN_KERNEL_TRANSPORT, [&] { return launch_transport_tiles<T>(a, c->tr_tile_ac, c->stream); });
    return prof(c, BFPN_KERNEL_TRANSPORT, [&] { return launch_transport<T>(a, c->tr_ac, c->stream); });
}

template <typename T>
cudaError_t enq_angle(bfpn_ctx* c, void* X, const void* fac, int ng = -1) {
    AngleArgs<T> a;
    a.F = as<T>(X);
    a.fac = as<const T>(const_cast<void*>(fac));
    a.sine_u = as<const T>(c->sine_u);
    a.sine_v = as<const T>(c->sine_v);
    a.Nom = c->Nom;
    a.Nmu = c->Nmu;
    a.nyz = c->nyz;
    a.Ng = ng >= 0 ? ng : c->Ng;
    a.slices_per_block = c->ang_slices;
    a.err = c->dev_err;
    a.pairs = c->tr_pairs ? 1 : 0;
    return prof(c, BFPN_KERNEL_ANGLE, [&] { return launch_angle<T>(a, c->stream); });
}

// The source from primary arrays P1, P2 of nyz positions (row stride
// nyz * NA) into S; A1 / A2 (and the tensor-core operand) in the context's
// A block, sized for those positions.  pread (may be null) is recorded once
// the last kernel that reads P1 and P2 has been enqueued.
template <typename T>
cudaError_t enq_source_on(bfpn_ctx* c, const void* P1, const void* P2, void* S, int nyz,
                          cudaEvent_t pread = nullptr) {
    SourceArgs<T> a;
    a.P1 = as<const T>(const_cast<void*>(P1));
    a.P2 = as<const T>(const_cast<void*>(P2));
    a.ker_v = as<const T>(c->ker_v);
    a.groups = c->groups;
    a.n_groups = c->n_groups;
    a.A1 = as<T>(c->A1);
    a.A2 = as<T>(c->A2);
    a.S = as<T>(S);
    a.e1 = c->e1;
    a.e2 = c->e2;
    a.tile_lo = c->tile_lo;
    a.tile_hi = c->tile_hi;
    a.Ng = c->Ng;
    a.nyz = nyz;
    a.NA = c->NA;
    a.dg = c->d.dg;
    const long long per_e = static_cast<long long>(nyz) * c->NA;
    cudaError_t e;
    if (sizeof(T) == sizeof(float) && c->use_umma && c->bblob && c->ablob && c->eblob) {
        // tensor cores: the angular stage writes the energy stage's split-bf16
        // operand into the A block, the energy stage reads it
        uint8_t* q = static_cast<uint8_t*>(c->A1);
        e = prof(c, BFPN_KERNEL_SOURCE_ANGULAR, [&] {
            return launch_source_angular_pipe(as<const float>(const_cast<void*>(P1)),
                                              as<const float>(const_cast<void*>(P2)),
                                              static_cast<uint8_t*>(c->ablob), static_cast<const uint8_t*>(c->bblob),
                                              c->groups, c->n_groups, q, c->Ng, c->dev_err, nyz, c->NA,
                                              c->umma_nt, c->umma_bk, c->umma_ntiles, c->ulist, c->ubegin,
                                              c->stream, pread, !c->src_prepacked);
        });
        if (e != cudaSuccess) return e;
        return prof(c, BFPN_KERNEL_SOURCE_ENERGY, [&] {
            return launch_source_energy_umma(q, static_cast<const uint8_t*>(c->eblob), c->ework, c->ework_begin,
                                             c->e_et, c->e_emax, as<float>(S), c->dev_err, per_e, c->Ng, c->stream);
        });
    }
    e = prof(c, BFPN_KERNEL_SOURCE_ANGULAR, [&] { return launch_source_angular<T>(a, c->stream); });
    if (e != cudaSuccess) return e;
    if (pread && (e = cudaEventRecord(pread, c->stream)) != cudaSuccess) return e;
    return prof(c, BFPN_KERNEL_SOURCE_ENERGY, [&] { return launch_source_energy<T>(a, c->tile_e, c->stream); });
}

template <typename T>
cudaError_t enq_source(bfpn_ctx* c, cudaEvent_t pread = nullptr) {
    return enq_source_on<T>(c, c->st[0][0], c->st[0][1], c->src, c->nyz, pread);
}

// transport half-step, angle full step, transport half-step on one array
// (the per-array part of stepPrimary/stepSecondary; the operations on F and
// f are independent, so each array runs its own T-A-T sequence).
template <typename T>
cudaError_t enq_tat(bfpn_ctx* c, int species, int coef, bool do_tr, bool do_an, bool preserve) {
    void* X = c->st[species][coef];
    const double h = 0.5 * c->d.dt;
    cudaError_t e = cudaSuccess;
    if (do_tr) {
        void* Y = transport_in_place(c) ? X : c->tmp;
        e = enq_transport<T>(c, X, Y, h, preserve);
        if (e != cudaSuccess) return e;
        if (do_an) {
            e = enq_angle<T>(c, Y, c->fac_step);
            if (e != cudaSuccess) return e;
        }
        return enq_transport<T>(c, Y, X, h, preserve);
    }
    if (do_an) e = enq_angle<T>(c, X, c->fac_step);
    return e;
}

// One depth step: the loop body of BFPnSolver::solve (bfpm_solver.cu:2201-2232).
// Lite-memory step (the lite branch of solve, bfpm_solver.cu:2191-2210):
// stepLitePrimary and computeIntegratedDepthDoseLite, proxy 0.
template <typename T>
cudaError_t enq_lite_step(bfpn_ctx* c) {
    const int trap = (c->p.flags & BFPN_FLAG_TRAPEZOIDAL_YZ) ? 1 : 0;
    const int n = lite_energy_grid(c->per_e);
    cudaError_t e = prof(c, BFPN_KERNEL_ENERGY, [&] {
        return launch_lite_energy<T>(as<T>(c->st[0][0]), c->lite_coef, c->d.dt, c->Ng, c->per_e, c->dose_coef, c->NA,
                                     c->Ny, c->Nz, trap, c->partials, c->stream);
    });
    if (e != cudaSuccess) return e;
    const double w = c->d.du * c->d.dv * c->d.dy * c->d.dz;
    return prof(c, BFPN_KERNEL_IDD, [&] {
        return launch_finalize_idd(c->partials, n, nullptr, 0, w, c->d.dg, c->hist_idd, c->hist_proxy, c->counter,
                                   c->hist_cap, 1, c->stream);
    });
}

// T-A-T of both arrays of a species: psi^1 on the context stream and, inside
// an overlapped body, psi^2 beside it on s_f[species] (the two chains share
// no array: the transport is in place there); one after the other elsewhere.
template <typename T>
cudaError_t enq_tat_pair(bfpn_ctx* c, int species, bool do_tr, bool do_an, bool preserve_F, bool preserve_f) {
    cudaError_t e;
    if (!c->split_tat) {
        if ((e = enq_tat<T>(c, species, 0, do_tr, do_an, preserve_F)) != cudaSuccess) return e;
        return enq_tat<T>(c, species, 1, do_tr, do_an, preserve_f);
    }
    cudaStream_t own = c->stream, side = c->s_f[species];
    if ((e = cudaEventRecord(c->ev_ff[species], own)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(side, c->ev_ff[species], 0)) != cudaSuccess) return e;
    c->stream = side;
    e = enq_tat<T>(c, species, 1, do_tr, do_an, preserve_f);
    c->stream = own;
    if (e != cudaSuccess) return e;
    if ((e = enq_tat<T>(c, species, 0, do_tr, do_an, preserve_F)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(c->ev_fj[species], side)) != cudaSuccess) return e;
    return cudaStreamWaitEvent(own, c->ev_fj[species], 0);
}

// IDD partial sums of the primary's last energy pass, by step parity (the
// secondary half of one step and the primary half of the next can be in
// flight together).
double* primary_partials(bfpn_ctx* c, int step) {
    return c->partials + ((step & 1) ? 4 : 0) * static_cast<size_t>(c->n_part);
}

// stepPrimary (bfpm_solver.cu:3238-3311) / stepPrimaryEnergyOnly (3313-3333),
// the last energy pass writing the IDD partials into partP.
template <typename T>
cudaError_t enq_primary_half(bfpn_ctx* c, double* partP) {
    const unsigned fl = c->p.flags;
    cudaError_t e;
    if ((e = enq_energy<T>(c, 0, c->ecoef_half, false, nullptr)) != cudaSuccess) return e;
    if (!(fl & BFPN_FLAG_ENERGY_ONLY)) {
        const bool do_tr = !(fl & BFPN_FLAG_NO_TRANSPORT), do_an = !(fl & BFPN_FLAG_NO_ANGLE);
        const bool clip_F = !(fl & BFPN_FLAG_NO_SPATIAL_CLIPPING);
        if ((e = enq_tat_pair<T>(c, 0, do_tr, do_an, !clip_F, true)) != cudaSuccess) return e;
    }
    return enq_energy<T>(c, 0, c->ecoef_half, false, partP);
}

template <typename T>
cudaError_t enq_finalize(bfpn_ctx* c, const double* partP, const double* partS, int nS) {
    const int nP = energy_grid(c->per_e, c->energy_block);
    const double w = c->d.du * c->d.dv * c->d.dy * c->d.dz;
    return prof(c, BFPN_KERNEL_IDD, [&] {
        return launch_finalize_idd(partP, nP, partS, nS, w, c->d.dg, c->hist_idd, c->hist_proxy, c->counter,
                                   c->hist_cap, 1, c->stream);
    });
}

// stepSecondary (3335-3394) and the step's IDD (partP from its primary
// half): the source depends only on the primary, which this half does not
// change, so both of the reference's evaluations are the same tensor; it is
// built once.  Transport of the secondary always clips F1 (3355-3356) and
// always runs.  pread: see enq_source_on.
template <typename T>
cudaError_t enq_secondary_half(bfpn_ctx* c, const double* partP, cudaEvent_t pread) {
    double* partS = c->partials + 2 * static_cast<size_t>(c->n_part);
    cudaError_t e;
    if ((e = enq_source<T>(c, pread)) != cudaSuccess) return e;
    if ((e = enq_energy<T>(c, 1, c->ecoef_half, true, nullptr)) != cudaSuccess) return e;
    if ((e = enq_tat_pair<T>(c, 1, true, true, false, true)) != cudaSuccess) return e;
    if ((e = enq_energy<T>(c, 1, c->ecoef_half, true, partS)) != cudaSuccess) return e;
    return enq_finalize<T>(c, partP, partS, energy_grid(c->per_e, c->energy_block));
}

// The IDD of a step without a secondary half (step 0, primary-only and
// energy-only runs): the secondary state's share, as it stands, unless it is
// known to be zero.
template <typename T>
cudaError_t enq_first_finalize(bfpn_ctx* c, const double* partP, bool secondary_zero) {
    const unsigned fl = c->p.flags;
    double* partS = c->partials + 2 * static_cast<size_t>(c->n_part);
    int nS = 0;
    if (!secondary_zero) {
        nS = idd_partials_grid(c->per_e);
        cudaError_t e = prof(c, BFPN_KERNEL_IDD, [&] {
            return launch_idd_partials<T>(as<const T>(c->st[1][0]), as<const T>(c->st[1][1]), c->dose_coef, c->Ng,
                                          c->per_e, c->NA, c->Ny, c->Nz, (fl & BFPN_FLAG_TRAPEZOIDAL_YZ) ? 1 : 0, 0,
                                          partS, nS, c->stream);
        });
        if (e != cudaSuccess) return e;
    }
    return enq_finalize<T>(c, partP, partS, nS);
}

template <typename T>
cudaError_t enq_step(bfpn_ctx* c, bool first, bool secondary_zero) {
    if (c->lite) return enq_lite_step<T>(c);
    const unsigned fl = c->p.flags;
    double* partP = primary_partials(c, c->steps_done);
    cudaError_t e;
    if ((e = enq_primary_half<T>(c, partP)) != cudaSuccess) return e;
    const bool secondary = !(fl & (BFPN_FLAG_ENERGY_ONLY | BFPN_FLAG_PRIMARY_ONLY)) && !first;
    if (secondary) return enq_secondary_half<T>(c, partP, nullptr);
    return enq_first_finalize<T>(c, partP, secondary_zero);
}

// Overlapped form of regular steps (one context stream, the secondary half on
// s_sec):
//   body(n) = [secondary half of step n-1 + its IDD] on s_sec, beside
//             [primary half of step n] on the context stream,
// where the primary's first kernel waits for the event recorded after the
// source's last read of the primary (the pack), and the body joins s_sec
// back before it ends.  The primary half of step n writes the partials of
// parity n while the secondary half of n-1 reads those of parity n-1.  Same
// kernels on the same inputs as the sequential order, so the same values.
template <typename T>
cudaError_t enq_overlap_body(bfpn_ctx* c, int step) {
    cudaError_t e;
    if ((e = cudaEventRecord(c->ev_fork, c->stream)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(c->s_sec, c->ev_fork, 0)) != cudaSuccess) return e;
    cudaStream_t main = c->stream;
    c->stream = c->s_sec;
    c->split_tat = c->split_chains;
    e = enq_secondary_half<T>(c, primary_partials(c, step - 1), c->ev_pread);
    c->stream = main;
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, c->ev_pread, 0);
    if (e == cudaSuccess) e = enq_primary_half<T>(c, primary_partials(c, step));
    c->split_tat = false;
    if (e != cudaSuccess) return e;
    if ((e = cudaEventRecord(c->ev_join, c->s_sec)) != cudaSuccess) return e;
    return cudaStreamWaitEvent(c->stream, c->ev_join, 0);
}

// ---- fused primary energy passes --------------------------------------------
// With the fused kernel (mixed precision, eq15 modes, transport in place) the
// steps of one bfpn_step call run as
//   open(n0) | body(n0+1) ... body(n0+k-1) | close(n0+k-1)
// where open(n) is the primary's opening energy pass and T-A-T of step n;
// body(n) = [energy_fused_kernel: the closing pass of step n-1 (its IDD
// partials and the source's operand) with the opening pass of step n, then
// the primary's T-A-T of step n] on the context stream, beside [the source of
// step n-1 from that operand (no pack pass), the secondary half of step n-1
// and its IDD] on s_sec; close(n) is the closing pass and secondary half of
// the call's last step.  Step 0 has no secondary half: body(1) finalises its
// IDD on the context stream.  Each kernel applies the unfused order's
// arithmetic to the same inputs, so the states are the same (a few values
// far below the peak aside, which may round one float step apart); a
// primary energy pass and the pack pass are saved per step.
bool fused_ok(const bfpn_ctx* c) {
    const unsigned fl = c->p.flags;
    if (!c->fuse_energy || !c->overlap || c->prec != BFPN_PREC_MIXED || c->lite || c->ooc ||
        !transport_in_place(c) || c->energy_block != 128)
        return false;
    if (fl & (BFPN_FLAG_ENERGY_ONLY | BFPN_FLAG_PRIMARY_ONLY | BFPN_FLAG_NO_TRANSPORT | BFPN_FLAG_NO_ANGLE |
              BFPN_FLAG_LEGACY_ENERGY))
        return false;
    const int mode = (fl & BFPN_FLAG_EQ15_STRAGGLING) ? EMODE_EQ15_STRAG : EMODE_EQ15;
    if (!energy_fused_supported(c->per_e, mode, c->NA)) return false;
    // the secondary's source must read the operand the fused kernel writes
    return c->n_groups == 0 || (c->use_umma && c->ablob && c->bblob && c->eblob);
}

cudaError_t enq_energy_fused(bfpn_ctx* c, double* partP) {
    EnergyFusedArgs A;
    EnergyArgs<float>& a = A.e;
    a.F = as<float>(c->st[0][0]);
    a.f = as<float>(c->st[0][1]);
    a.src = nullptr;
    a.coef = c->ecoef_half;
    a.Ng = c->Ng;
    a.lanes = c->per_e;
    a.mode = (c->p.flags & BFPN_FLAG_EQ15_STRAGGLING) ? EMODE_EQ15_STRAG : EMODE_EQ15;
    a.partials = partP;
    a.dose_coef = c->dose_coef;
    a.NA = c->NA;
    a.Ny = c->Ny;
    a.Nz = c->Nz;
    a.trapezoidal = (c->p.flags & BFPN_FLAG_TRAPEZOIDAL_YZ) ? 1 : 0;
    A.ablob = c->n_groups > 0 ? static_cast<uint8_t*>(c->ablob) : nullptr;
    A.gmap = c->gmap;
    A.n_mt = (c->nyz + 63) / 64;
    A.nk = (c->NA + c->umma_bk - 1) / c->umma_bk;
    return prof(c, BFPN_KERNEL_ENERGY_FUSED, [&] { return launch_energy_fused(A, c->stream); });
}

// The primary's opening energy pass and T-A-T of step steps_done.
cudaError_t enq_primary_open(bfpn_ctx* c) {
    cudaError_t e = enq_energy<float>(c, 0, c->ecoef_half, false, nullptr);
    if (e != cudaSuccess) return e;
    const bool clip_F = !(c->p.flags & BFPN_FLAG_NO_SPATIAL_CLIPPING);
    return enq_tat_pair<float>(c, 0, true, true, !clip_F, true);
}

// body(step): see above; first_prev = step-1 is step 0.
cudaError_t enq_fused_body(bfpn_ctx* c, int step, bool first_prev) {
    double* partP = primary_partials(c, step - 1);
    const bool clip_F = !(c->p.flags & BFPN_FLAG_NO_SPATIAL_CLIPPING);
    cudaError_t e = enq_energy_fused(c, partP);
    if (e != cudaSuccess) return e;
    if (first_prev) {
        if ((e = enq_first_finalize<float>(c, partP, c->secondary_zero)) != cudaSuccess) return e;
        c->split_tat = c->split_chains;
        e = enq_tat_pair<float>(c, 0, true, true, !clip_F, true);
        c->split_tat = false;
        return e;
    }
    if (c->profiling) {  // per-kernel timing: one kernel after the other
        c->src_prepacked = true;
        e = enq_secondary_half<float>(c, partP, nullptr);
        c->src_prepacked = false;
        return e == cudaSuccess ? enq_tat_pair<float>(c, 0, true, true, !clip_F, true) : e;
    }
    cudaStream_t main = c->stream;
    if ((e = cudaEventRecord(c->ev_fork, main)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(c->s_sec, c->ev_fork, 0)) != cudaSuccess) return e;
    c->stream = c->s_sec;
    c->split_tat = c->split_chains;
    c->src_prepacked = true;
    e = enq_secondary_half<float>(c, partP, nullptr);
    c->src_prepacked = false;
    c->stream = main;
    if (e == cudaSuccess) e = enq_tat_pair<float>(c, 0, true, true, !clip_F, true);
    c->split_tat = false;
    if (e != cudaSuccess) return e;
    if ((e = cudaEventRecord(c->ev_join, c->s_sec)) != cudaSuccess) return e;
    return cudaStreamWaitEvent(c->stream, c->ev_join, 0);
}

// close: the owed closing pass and secondary half (or step-0 IDD) of step steps_done-1.
cudaError_t enq_fused_close(bfpn_ctx* c) {
    double* partP = primary_partials(c, c->steps_done - 1);
    cudaError_t e = enq_energy<float>(c, 0, c->ecoef_half, false, partP);
    if (e != cudaSuccess) return e;
    if (c->pending_first) return enq_first_finalize<float>(c, partP, c->secondary_zero);
    return enq_secondary_half<float>(c, partP, nullptr);
}

cudaError_t enq_step_any(bfpn_ctx* c, bool first, bool secondary_zero) {
    return c->prec == BFPN_PREC_FP64 ? enq_step<double>(c, first, secondary_zero)
                                     : enq_step<float>(c, first, secondary_zero);
}

// ---------------------------------------------------------------------------
// Out-of-core mode (BFPN_FLAG_STREAMING_FULL; the reference's
// solveStreamingFull, bfpm_solver.cu:3113-3236, with its backing files
// replaced by pinned host memory).  The operators split two ways: the energy
// sweep and the source are local to a lane (position, angle), so they run on
// lane chunks -- every group of lc_pos whole positions, moved with 2D copies
// (rows of lc lanes on the device; a partial last chunk is zero-padded, and
// zeros stay zero and add nothing to the IDD); transport and angular
// diffusion are local to a group, so they run on group chunks of ecg
// contiguous groups.  A depth step is the in-core step's operator sequence,
// each operator one streamed pass; the kernels are the in-core ones.  The
// secondary's source is rebuilt for each lane chunk from the primary in both
// of its energy passes (the primary does not change in between).
// ---------------------------------------------------------------------------
bfpn_status ensure_ooc(bfpn_ctx* c) {
    const int lc_pos = std::max(1, std::min(c->nyz, c->ooc_lane_req / c->NA));
    const int ecg = std::max(1, std::min(c->Ng, c->ooc_group_req));
    if (c->ooc_ready && lc_pos == c->lc_pos && ecg == c->ecg) return BFPN_OK;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (!c->s_in) {
        CUDA_TRY(c, cudaStreamCreateWithFlags(&c->s_in, cudaStreamNonBlocking));
        CUDA_TRY(c, cudaStreamCreateWithFlags(&c->s_out, cudaStreamNonBlocking));
        for (int k = 0; k < 2; ++k) {
            CUDA_TRY(c, cudaEventCreateWithFlags(&c->ev_in[k], cudaEventDisableTiming));
            CUDA_TRY(c, cudaEventCreateWithFlags(&c->ev_comp[k], cudaEventDisableTiming));
            CUDA_TRY(c, cudaEventCreateWithFlags(&c->ev_out[k], cudaEventDisableTiming));
        }
        CUDA_TRY(c, cudaEventCreateWithFlags(&c->ev_pass, cudaEventDisableTiming));
    }
    CUDA_TRY(c, cudaStreamSynchronize(c->s_in));
    CUDA_TRY(c, cudaStreamSynchronize(c->s_out));
    for (auto& slot : c->dl)
        for (void*& p : slot) dfree(c, p);
    for (void*& p : c->dgc) dfree(c, p);
    dfree(c, c->tmp);
    dfree(c, c->src);
    dfree(c, c->A1);
    c->A2 = nullptr;
    dfree(c, c->ablob);
    dfree(c, c->ooc_part);
    c->ooc_ready = false;
    c->lc_pos = lc_pos;
    c->lc = lc_pos * c->NA;
    c->n_lc = (c->nyz + lc_pos - 1) / lc_pos;
    c->ecg = ecg;
    const size_t lane_arr = static_cast<size_t>(c->Ng) * c->lc * c->elem;
    const size_t group_arr = static_cast<size_t>(ecg) * c->per_e * c->elem;
    const bool secondary = !(c->p.flags & (BFPN_FLAG_PRIMARY_ONLY | BFPN_FLAG_ENERGY_ONLY));
    bfpn_status s;
    for (auto& slot : c->dl)
        for (int k = 0; k < (secondary ? 4 : 2); ++k)
            if ((s = dalloc(c, &slot[k], lane_arr)) != BFPN_OK) return s;
    for (void*& p : c->dgc)
        if ((s = dalloc(c, &p, group_arr)) != BFPN_OK) return s;
    if (!c->tr_inplace && (s = dalloc(c, &c->tmp, group_arr)) != BFPN_OK) return s;
    if (secondary) {
        if ((s = dalloc(c, &c->src, lane_arr)) != BFPN_OK) return s;
        c->a_bytes = c->prec == BFPN_PREC_MIXED ? std::max(2 * lane_arr, umma_q_bytes(c->lc, c->Ng)) : 2 * lane_arr;
        if ((s = dalloc(c, &c->A1, c->a_bytes)) != BFPN_OK) return s;
        c->A2 = static_cast<char*>(c->A1) + lane_arr;
        CUDA_TRY(c, cudaMemsetAsync(c->A1, 0, c->a_bytes, c->stream));
        if (c->prec == BFPN_PREC_MIXED && c->bblob && c->n_groups > 0) {
            void* ab = nullptr;
            if (dalloc(c, &ab, umma_pack_bytes(c->n_groups, lc_pos, c->NA, c->umma_bk)) == BFPN_OK) c->ablob = ab;
            else cudaGetLastError();  // without it the source stays on the CUDA-core kernels
        }
    }
    const size_t part = 4 * static_cast<size_t>(c->n_lc) * energy_grid(c->lc, c->energy_block);
    if ((s = dalloc(c, &c->ooc_part, part * sizeof(double))) != BFPN_OK) return s;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->ooc_ready = true;
    return BFPN_OK;
}

// Lane chunk k of host array H to / from device rows of lc lanes.
cudaError_t ooc_lane_copy(bfpn_ctx* c, void* H, void* D, int k, bool to_device, cudaStream_t st) {
    const size_t e = c->elem, pitch_h = static_cast<size_t>(c->per_e) * e, pitch_d = static_cast<size_t>(c->lc) * e;
    const long long p0 = static_cast<long long>(k) * c->lc_pos;
    const size_t lanes = static_cast<size_t>(std::min<long long>(c->lc_pos, c->nyz - p0)) * c->NA;
    char* h = static_cast<char*>(H) + p0 * c->NA * e;
    cudaError_t r;
    if (!to_device) return cudaMemcpy2DAsync(h, pitch_h, D, pitch_d, lanes * e, c->Ng, cudaMemcpyDeviceToHost, st);
    r = cudaMemcpy2DAsync(D, pitch_d, h, pitch_h, lanes * e, c->Ng, cudaMemcpyHostToDevice, st);
    if (r == cudaSuccess && lanes < static_cast<size_t>(c->lc))
        r = cudaMemset2DAsync(static_cast<char*>(D) + lanes * e, pitch_d, 0, (c->lc - lanes) * e, c->Ng, st);
    return r;
}

// The next pass reads host arrays this pass writes: both the copy-in and the
// compute stream wait for every copy out of this pass.
cudaError_t ooc_pass_end(bfpn_ctx* c) {
    cudaError_t e = cudaEventRecord(c->ev_pass, c->s_out);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->s_in, c->ev_pass, 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, c->ev_pass, 0);
    return e;
}

// One energy half-step of a species over every lane chunk; with partials,
// energy_grid(lc) partial pairs per chunk, chunk after chunk (*count in total).
template <typename T>
cudaError_t ooc_energy_pass(bfpn_ctx* c, int species, bool with_source, double* partials, int* count) {
    const int gpc = energy_grid(c->lc, c->energy_block);
    cudaError_t e;
    for (int k = 0; k < c->n_lc; ++k) {
        const int sl = k & 1;
        void* const* B = c->dl[sl];
        // in: once the copies out of this slot's previous chunk are done
        if ((e = cudaStreamWaitEvent(c->s_in, c->ev_out[sl], 0)) != cudaSuccess) return e;
        if ((e = ooc_lane_copy(c, c->st[species][0], B[0], k, true, c->s_in)) != cudaSuccess) return e;
        if ((e = ooc_lane_copy(c, c->st[species][1], B[1], k, true, c->s_in)) != cudaSuccess) return e;
        if (with_source) {
            if ((e = ooc_lane_copy(c, c->st[0][0], B[2], k, true, c->s_in)) != cudaSuccess) return e;
            if ((e = ooc_lane_copy(c, c->st[0][1], B[3], k, true, c->s_in)) != cudaSuccess) return e;
        }
        if ((e = cudaEventRecord(c->ev_in[sl], c->s_in)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(c->stream, c->ev_in[sl], 0)) != cudaSuccess) return e;
        if (with_source && (e = enq_source_on<T>(c, B[2], B[3], c->src, c->lc_pos)) != cudaSuccess) return e;
        EnergyArgs<T> a;
        a.F = as<T>(B[0]);
        a.f = as<T>(B[1]);
        a.src = with_source ? as<const T>(c->src) : nullptr;
        a.coef = c->ecoef_half;
        a.Ng = c->Ng;
        a.lanes = c->lc;
        a.lane0 = static_cast<long long>(k) * c->lc;
        if (c->p.flags & BFPN_FLAG_LEGACY_ENERGY) a.mode = EMODE_LEGACY;
        else if (c->p.flags & BFPN_FLAG_EQ15_STRAGGLING) a.mode = EMODE_EQ15_STRAG;
        else a.mode = EMODE_EQ15;
        a.partials = partials ? partials + 2 * static_cast<size_t>(k) * gpc : nullptr;
        a.dose_coef = c->dose_coef;
        a.NA = c->NA;
        a.Ny = c->Ny;
        a.Nz = c->Nz;
        a.trapezoidal = (c->p.flags & BFPN_FLAG_TRAPEZOIDAL_YZ) ? 1 : 0;
        if ((e = prof(c, BFPN_KERNEL_ENERGY, [&] { return launch_energy<T>(a, c->energy_block, c->stream); })) !=
            cudaSuccess)
            return e;
        // out: after the chunk's kernels
        if ((e = cudaEventRecord(c->ev_comp[sl], c->stream)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(c->s_out, c->ev_comp[sl], 0)) != cudaSuccess) return e;
        if ((e = ooc_lane_copy(c, c->st[species][0], B[0], k, false, c->s_out)) != cudaSuccess) return e;
        if ((e = ooc_lane_copy(c, c->st[species][1], B[1], k, false, c->s_out)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(c->ev_out[sl], c->s_out)) != cudaSuccess) return e;
    }
    if (count) *count = c->n_lc * gpc;
    return ooc_pass_end(c);
}

// Transport half-step, angle step, transport half-step on one array, group chunk by group chunk.
template <typename T>
cudaError_t ooc_tat_pass(bfpn_ctx* c, int species, int coef, bool do_tr, bool do_an, bool preserve) {
    const double h = 0.5 * c->d.dt;
    char* X = static_cast<char*>(c->st[species][coef]);
    const size_t row = static_cast<size_t>(c->per_e) * c->elem;
    cudaError_t e;
    int k = 0;
    for (int e0 = 0; e0 < c->Ng; e0 += c->ecg, ++k) {
        const int g = std::min(c->ecg, c->Ng - e0), sl = k & 1;
        void* D = c->dgc[sl];
        const void* fac = static_cast<const char*>(c->fac_step) + static_cast<size_t>(e0) * c->NA * c->elem;
        if ((e = cudaStreamWaitEvent(c->s_in, c->ev_out[sl], 0)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(D, X + e0 * row, g * row, cudaMemcpyHostToDevice, c->s_in)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(c->ev_in[sl], c->s_in)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(c->stream, c->ev_in[sl], 0)) != cudaSuccess) return e;
        if (do_tr) {
            void* Y = transport_in_place(c) ? D : c->tmp;
            if ((e = enq_transport<T>(c, D, Y, h, preserve, g)) != cudaSuccess) return e;
            if (do_an && (e = enq_angle<T>(c, Y, fac, g)) != cudaSuccess) return e;
            if ((e = enq_transport<T>(c, Y, D, h, preserve, g)) != cudaSuccess) return e;
        } else if (do_an) {
            if ((e = enq_angle<T>(c, D, fac, g)) != cudaSuccess) return e;
        }
        if ((e = cudaEventRecord(c->ev_comp[sl], c->stream)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(c->s_out, c->ev_comp[sl], 0)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(X + e0 * row, D, g * row, cudaMemcpyDeviceToHost, c->s_out)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(c->ev_out[sl], c->s_out)) != cudaSuccess) return e;
    }
    return ooc_pass_end(c);
}

// One depth step: enq_step's operator sequence, streamed.
template <typename T>
cudaError_t ooc_step(bfpn_ctx* c, bool first, bool secondary_zero) {
    const unsigned fl = c->p.flags;
    const bool energy_only = fl & BFPN_FLAG_ENERGY_ONLY;
    const bool do_tr = !(fl & BFPN_FLAG_NO_TRANSPORT), do_an = !(fl & BFPN_FLAG_NO_ANGLE);
    const size_t half = 2 * static_cast<size_t>(c->n_lc) * energy_grid(c->lc, c->energy_block);
    double* partP = static_cast<double*>(c->ooc_part);
    double* partS = partP + half;
    int nP = 0, nS = 0;
    cudaError_t e;
    if ((e = ooc_energy_pass<T>(c, 0, false, nullptr, nullptr)) != cudaSuccess) return e;
    if (!energy_only) {
        const bool clip_F = !(fl & BFPN_FLAG_NO_SPATIAL_CLIPPING);
        if ((e = ooc_tat_pass<T>(c, 0, 0, do_tr, do_an, !clip_F)) != cudaSuccess) return e;
        if ((e = ooc_tat_pass<T>(c, 0, 1, do_tr, do_an, true)) != cudaSuccess) return e;
    }
    if ((e = ooc_energy_pass<T>(c, 0, false, partP, &nP)) != cudaSuccess) return e;
    const bool secondary = !energy_only && !(fl & BFPN_FLAG_PRIMARY_ONLY) && !first;
    if (secondary) {
        if ((e = ooc_energy_pass<T>(c, 1, true, nullptr, nullptr)) != cudaSuccess) return e;
        if ((e = ooc_tat_pass<T>(c, 1, 0, true, true, false)) != cudaSuccess) return e;
        if ((e = ooc_tat_pass<T>(c, 1, 1, true, true, true)) != cudaSuccess) return e;
        if ((e = ooc_energy_pass<T>(c, 1, true, partS, &nS)) != cudaSuccess) return e;
    } else if (!secondary_zero) {
        return cudaErrorNotSupported;  // an uploaded secondary that this step does not advance
    }
    const double w = c->d.du * c->d.dv * c->d.dy * c->d.dz;
    return prof(c, BFPN_KERNEL_IDD, [&] {
        return launch_finalize_idd(partP, nP, partS, nS, w, c->d.dg, c->hist_idd, c->hist_proxy, c->counter,
                                   c->hist_cap, 1, c->stream);
    });
}

bfpn_status ensure_history(bfpn_ctx* c, int needed) {
    if (needed <= c->hist_cap) return BFPN_OK;
    int cap = c->hist_cap;
    while (cap < needed) cap *= 2;
    void *ni = nullptr, *np = nullptr;
    bfpn_status s;
    if ((s = dalloc(c, &ni, cap * sizeof(double))) != BFPN_OK) return s;
    if ((s = dalloc(c, &np, cap * sizeof(double))) != BFPN_OK) return s;
    CUDA_TRY(c, cudaMemcpyAsync(ni, c->hist_idd, c->hist_cap * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(np, c->hist_proxy, c->hist_cap * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    // the step graphs hold the old addresses: drop them before the old buffers go
    drop_graphs(c);
    void* old_idd = c->hist_idd;
    void* old_proxy = c->hist_proxy;
    dfree(c, old_idd);
    dfree(c, old_proxy);
    c->hist_idd = static_cast<double*>(ni);
    c->hist_proxy = static_cast<double*>(np);
    c->hist_cap = cap;
    return BFPN_OK;
}

// Regular steps of this context may overlap: graphs on, the standard
// operator set, transport in place (no shared scratch array).
bool overlap_ok(const bfpn_ctx* c) {
    const unsigned fl = c->p.flags;
    return c->overlap && c->use_graphs && !c->lite && !c->ooc && transport_in_place(c) &&
           !(fl & (BFPN_FLAG_ENERGY_ONLY | BFPN_FLAG_PRIMARY_ONLY | BFPN_FLAG_NO_TRANSPORT | BFPN_FLAG_NO_ANGLE));
}

bfpn_status ensure_overlap_objects(bfpn_ctx* c) {
    if (c->s_sec) return BFPN_OK;
    CUDA_TRY(c, cudaStreamCreateWithFlags(&c->s_sec, cudaStreamNonBlocking));
    for (cudaStream_t* st : {&c->s_f[0], &c->s_f[1]}) CUDA_TRY(c, cudaStreamCreateWithFlags(st, cudaStreamNonBlocking));
    for (cudaEvent_t* e : {&c->ev_fork, &c->ev_pread, &c->ev_join, &c->ev_ff[0], &c->ev_ff[1], &c->ev_fj[0], &c->ev_fj[1]})
        CUDA_TRY(c, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    return BFPN_OK;
}

// The owed secondary half of step steps_done-1, enqueued on the context stream.
bfpn_status flush_secondary(bfpn_ctx* c) {
    if (!c->pending_sec) return BFPN_OK;
    c->pending_sec = false;
    const double* partP = primary_partials(c, c->steps_done - 1);
    if (c->prec == BFPN_PREC_FP64) CUDA_TRY(c, enq_secondary_half<double>(c, partP, nullptr));
    else CUDA_TRY(c, enq_secondary_half<float>(c, partP, nullptr));
    return BFPN_OK;
}

// One overlapped regular step (step = steps_done): the primary half alone
// when no secondary half is owed, else the captured body of its parity.
bfpn_status overlap_step(bfpn_ctx* c) {
    const int step = c->steps_done;
    if (!c->pending_sec) {
        double* partP = primary_partials(c, step);
        if (c->prec == BFPN_PREC_FP64) CUDA_TRY(c, enq_primary_half<double>(c, partP));
        else CUDA_TRY(c, enq_primary_half<float>(c, partP));
        c->pending_sec = true;
        return BFPN_OK;
    }
    cudaGraphExec_t& g = c->ovl_exec[step & 1];
    if (!g) {
        cudaGraph_t graph = nullptr;
        CUDA_TRY(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        const long long before = c->launches;
        cudaError_t ce = c->prec == BFPN_PREC_FP64 ? enq_overlap_body<double>(c, step) : enq_overlap_body<float>(c, step);
        c->kernels_per_step = static_cast<int>(c->launches - before);
        cudaError_t ee = cudaStreamEndCapture(c->stream, &graph);
        if (ce != cudaSuccess || ee != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            return fail(c, BFPN_CUDA_ERROR,
                        std::string("step capture failed: ") + cudaGetErrorString(ce != cudaSuccess ? ce : ee));
        }
        ce = cudaGraphInstantiate(&g, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) return fail(c, BFPN_CUDA_ERROR, std::string("graph instantiate: ") + cudaGetErrorString(ce));
    }
    CUDA_TRY(c, cudaGraphLaunch(g, c->stream));
    return BFPN_OK;
}

// One step of the fused order (step = steps_done); see enq_fused_body.
bfpn_status fused_step(bfpn_ctx* c) {
    const int step = c->steps_done;
    if (!c->pending_close) {
        CUDA_TRY(c, enq_primary_open(c));
        c->pending_close = true;
        c->pending_first = step == 0;
        return BFPN_OK;
    }
    if (c->pending_first || !c->use_graphs) {  // the body after step 0 runs once: no graph
        const long long before = c->launches;
        CUDA_TRY(c, enq_fused_body(c, step, c->pending_first));
        if (!c->pending_first) c->kernels_per_step = static_cast<int>(c->launches - before);
        c->pending_first = false;
        return BFPN_OK;
    }
    cudaGraphExec_t& g = c->fus_exec[step & 1];
    if (!g) {
        cudaGraph_t graph = nullptr;
        CUDA_TRY(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        const long long before = c->launches;
        cudaError_t ce = enq_fused_body(c, step, false);
        c->kernels_per_step = static_cast<int>(c->launches - before);
        cudaError_t ee = cudaStreamEndCapture(c->stream, &graph);
        if (ce != cudaSuccess || ee != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            return fail(c, BFPN_CUDA_ERROR,
                        std::string("step capture failed: ") + cudaGetErrorString(ce != cudaSuccess ? ce : ee));
        }
        ce = cudaGraphInstantiate(&g, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) return fail(c, BFPN_CUDA_ERROR, std::string("graph instantiate: ") + cudaGetErrorString(ce));
    }
    CUDA_TRY(c, cudaGraphLaunch(g, c->stream));
    return BFPN_OK;
}

bfpn_status flush_close(bfpn_ctx* c) {
    if (!c->pending_close) return BFPN_OK;
    c->pending_close = false;
    CUDA_TRY(c, enq_fused_close(c));
    c->pending_first = false;
    return BFPN_OK;
}

bfpn_status run_steps(bfpn_ctx* c, int nsteps) {
    if (!c->tables_loaded) return fail(c, BFPN_NOT_READY, "tables not loaded (bfpn_load_tables)");
    if (!c->beam_ready) return fail(c, BFPN_NOT_READY, "beam not initialised (bfpn_init_beam)");
    if (nsteps < 0) return fail(c, BFPN_INVALID_ARG, "nsteps < 0");
    bfpn_status s = ensure_history(c, c->steps_done + nsteps);
    if (s != BFPN_OK) return s;
    if (c->ooc) {  // streamed steps, launched eagerly
        if ((s = ensure_ooc(c)) != BFPN_OK) return s;
        for (int i = 0; i < nsteps; ++i) {
            const bool first = c->steps_done == 0;
            const long long before = c->launches;
            const cudaError_t e = c->prec == BFPN_PREC_FP64 ? ooc_step<double>(c, first, c->secondary_zero)
                                                            : ooc_step<float>(c, first, c->secondary_zero);
            if (e == cudaErrorNotSupported)
                return fail(c, BFPN_INVALID_ARG,
                            "out-of-core mode: an uploaded secondary state that a step does not advance");
            CUDA_TRY(c, e);
            c->kernels_per_step = static_cast<int>(c->launches - before);
            if (!first && !(c->p.flags & (BFPN_FLAG_ENERGY_ONLY | BFPN_FLAG_PRIMARY_ONLY))) c->secondary_zero = false;
            c->steps_done++;
        }
        return BFPN_OK;
    }
    const bool fus = fused_ok(c);
    const bool ovl = overlap_ok(c);
    if ((fus || ovl) && (s = ensure_overlap_objects(c)) != BFPN_OK) return s;
    for (int i = 0; i < nsteps; ++i) {
        const bool first = c->steps_done == 0;
        const bool secondary_stepping =
            !first && !(c->p.flags & (BFPN_FLAG_ENERGY_ONLY | BFPN_FLAG_PRIMARY_ONLY));
        if (fus) {
            if ((s = fused_step(c)) != BFPN_OK) return s;
        } else if (ovl && !first) {
            if ((s = overlap_step(c)) != BFPN_OK) return s;
        } else if (first || !c->use_graphs) {
            const long long before = c->launches;
            CUDA_TRY(c, enq_step_any(c, first, c->secondary_zero));
            if (!first) c->kernels_per_step = static_cast<int>(c->launches - before);
        } else {
            const int key = c->secondary_zero ? 1 : 0;
            if (!c->graph_exec || c->graph_key != key) {
                if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
                c->graph_exec = nullptr;
                cudaGraph_t graph = nullptr;
                CUDA_TRY(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
                const long long before = c->launches;
                cudaError_t ce = enq_step_any(c, false, c->secondary_zero);
                c->kernels_per_step = static_cast<int>(c->launches - before);
                cudaError_t ee = cudaStreamEndCapture(c->stream, &graph);
                if (ce != cudaSuccess || ee != cudaSuccess) {
                    if (graph) cudaGraphDestroy(graph);
                    cudaGetLastError();
                    return fail(c, BFPN_CUDA_ERROR,
                                std::string("step capture failed: ") +
                                    cudaGetErrorString(ce != cudaSuccess ? ce : ee));
                }
                ce = cudaGraphInstantiate(&c->graph_exec, graph, 0);
                cudaGraphDestroy(graph);
                if (ce != cudaSuccess) return fail(c, BFPN_CUDA_ERROR, std::string("graph instantiate: ") + cudaGetErrorString(ce));
                c->graph_key = key;
            }
            CUDA_TRY(c, cudaGraphLaunch(c->graph_exec, c->stream));
        }
        if (secondary_stepping) c->secondary_zero = false;
        c->steps_done++;
    }
    // every call leaves whole steps behind it
    if ((s = flush_close(c)) != BFPN_OK) return s;
    return flush_secondary(c);
}

template <typename T>
bfpn_status download_as(bfpn_ctx* c, const void* dev, double* host, size_t n) {
    if (sizeof(T) == sizeof(double)) {
        CUDA_TRY(c, cudaMemcpyAsync(host, dev, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        return BFPN_OK;
    }
    std::vector<T> tmp(n);
    CUDA_TRY(c, cudaMemcpyAsync(tmp.data(), dev, n * sizeof(T), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i < n; ++i) host[i] = static_cast<double>(tmp[i]);
    return BFPN_OK;
}


// Reads and clears the device error word that kernels with bounded waits set
// when a wait ran out (the stream must be idle).
bfpn_status check_device_error(bfpn_ctx* c) {
    if (!c->dev_err) return BFPN_OK;
    int h = 0;
    CUDA_TRY(c, cudaMemcpy(&h, c->dev_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h == 0) return BFPN_OK;
    CUDA_TRY(c, cudaMemsetAsync(c->dev_err, 0, sizeof(int), c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return fail(c, BFPN_TIMEOUT, "a bounded device wait ran out (code " + std::to_string(h) + "); results of the step are invalid");
}

struct TableView {
    const double* data;
    size_t size;
    bool known;
};

template <typename V>
TableView view_of(const V& v) {
    return TableView{v.data(), v.size(), true};
}

// known == false for an unknown table id
TableView table_of(const BeamTables& T, int which, std::vector<double>& tmp) {
    switch (which) {
        case BFPN_TABLE_S_S: return view_of(T.S_s);
        case BFPN_TABLE_T_C: return view_of(T.T_c);
        case BFPN_TABLE_SIG_TRG: return view_of(T.sig_trg);
        case BFPN_TABLE_SIGMA_C: return view_of(T.sigma);
        case BFPN_TABLE_EN: return view_of(T.en);
        case BFPN_TABLE_OMEND: return view_of(T.omega);
        case BFPN_TABLE_KER_E1: return view_of(T.ker_e1);
        case BFPN_TABLE_KER_E2: return view_of(T.ker_e2);
        case BFPN_TABLE_KER_V: return view_of(T.ker_v);
        case BFPN_TABLE_BAND:
            tmp.resize(2 * static_cast<size_t>(T.Ng));
            for (int i = 0; i < T.Ng; ++i) {
                tmp[2 * i] = T.band_begin[i];
                tmp[2 * i + 1] = T.band_end[i];
            }
            return view_of(tmp);
        case BFPN_TABLE_BEAM_YZA: return view_of(T.beam_yza);
        case BFPN_TABLE_BEAM_E: return view_of(T.beam_e);
        default: return TableView{nullptr, 0, false};
    }
}

bfpn_status set_device(bfpn_ctx* c) {
    CUDA_TRY(c, cudaSetDevice(c->device));
    return BFPN_OK;
}

}  // namespace

// ============================================================================
// C ABI
// ============================================================================
void bfpn::set_context_free_error(const std::string& msg) { g_create_error = msg; }

extern "C" {

const char* bfpn_version(void) { return "bfpn-b200 0.1.0 (sm_100a)"; }

const char* bfpn_status_string(bfpn_status s) {
    switch (s) {
        case BFPN_OK: return "ok";
        case BFPN_INVALID_ARG: return "invalid argument";
        case BFPN_OOM: return "out of device memory";
        case BFPN_CUDA_ERROR: return "CUDA error";
        case BFPN_TIMEOUT: return "timeout";
        case BFPN_IO_ERROR: return "I/O error";
        case BFPN_NOT_READY: return "not ready";
        case BFPN_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

const char* bfpn_last_error(const bfpn_ctx* ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

bfpn_status bfpn_read_tables(const char* data_path, int32_t Ng, double* mu, int32_t* mu_rows, double* sigma_c,
                             int32_t* sigma_rows) {
    if (!data_path || !mu || !mu_rows || !sigma_c || !sigma_rows || Ng <= 0)
        return fail(nullptr, BFPN_INVALID_ARG, "null argument or Ng <= 0");
    std::vector<double> m, s;
    int mr = 0, sr = 0;
    std::string path, err;
    if (!read_table_files(data_path, Ng, m, mr, s, sr, path, err)) return fail(nullptr, BFPN_IO_ERROR, err);
    std::memcpy(mu, m.data(), m.size() * sizeof(double));
    std::memcpy(sigma_c, s.data(), s.size() * sizeof(double));
    *mu_rows = mr;
    *sigma_rows = sr;
    return BFPN_OK;
}

bfpn_status bfpn_host_table(const bfpn_grid* grid, const bfpn_phys* phys, const double* mu, int32_t mu_rows,
                            const double* sigma_c, int32_t sigma_rows, int32_t which, double* out, uint64_t n,
                            uint64_t* n_out) {
    if (!grid || !phys || !sigma_c || !n_out || (!out && n > 0) || (!mu && mu_rows > 0))
        return fail(nullptr, BFPN_INVALID_ARG, "null argument");
    std::string why;
    if (!valid_grid(*grid, why)) return fail(nullptr, BFPN_INVALID_ARG, why);
    BeamTables T;
    if (!build_tables(*grid, *phys, mu, mu_rows, sigma_c, sigma_rows, T, why)) return fail(nullptr, BFPN_INVALID_ARG, why);
    std::vector<double> tmp;
    const TableView src = table_of(T, which, tmp);
    if (!src.known) return fail(nullptr, BFPN_INVALID_ARG, "unknown table id");
    *n_out = src.size;
    if (src.size > n) return fail(nullptr, BFPN_INVALID_ARG, "output buffer too small for the table");
    if (src.size) std::memcpy(out, src.data, src.size * sizeof(double));
    return BFPN_OK;
}

bfpn_status bfpn_footprint_bytes(const bfpn_grid* grid, const bfpn_phys* phys, int precision, uint64_t* bytes) {
    if (!grid || !bytes) return fail(nullptr, BFPN_INVALID_ARG, "null argument");
    std::string why;
    if (!valid_grid(*grid, why)) return fail(nullptr, BFPN_INVALID_ARG, why);
    if (precision != BFPN_PREC_FP64 && precision != BFPN_PREC_MIXED)
        return fail(nullptr, BFPN_INVALID_ARG, "unknown precision");
    if (phys && (phys->flags & BFPN_FLAG_STREAMING_FULL)) {  // device bytes at the default chunk sizes
        const size_t elem = precision == BFPN_PREC_FP64 ? 8 : 4;
        const long long nyz = static_cast<long long>(grid->Ny + 1) * (grid->Nz + 1), NA = grid->Nmu * grid->Nom;
        const long long lc = std::max<long long>(1, std::min<long long>(nyz, 262144 / NA)) * NA;
        const size_t lane_arr = static_cast<size_t>(grid->Ng) * lc * elem;
        const size_t group_arr = static_cast<size_t>(std::min(grid->Ng, 128)) * nyz * NA * elem;
        *bytes = 8 * lane_arr + 2 * group_arr + static_cast<size_t>(grid->Ng) * NA * NA * elem +
                 2 * static_cast<size_t>(grid->Ng) * grid->Ng * sizeof(double) + (64u << 20);
        return BFPN_OK;
    }
    *bytes = footprint(*grid, precision, phys && (phys->flags & BFPN_FLAG_LITE_MEMORY));
    return BFPN_OK;
}

bfpn_status bfpn_create(const bfpn_grid* grid, const bfpn_phys* phys, int precision, int device, bfpn_ctx** out) {
    if (!grid || !phys || !out) return fail(nullptr, BFPN_INVALID_ARG, "null argument");
    *out = nullptr;
    std::string why;
    if (!valid_grid(*grid, why)) return fail(nullptr, BFPN_INVALID_ARG, why);
    if (precision != BFPN_PREC_FP64 && precision != BFPN_PREC_MIXED)
        return fail(nullptr, BFPN_INVALID_ARG, "unknown precision");
    if (!(phys->density > 0) || !(phys->energy_density > 0) || !(phys->sig_E > 0))
        return fail(nullptr, BFPN_INVALID_ARG, "density and sigma_E must be positive");
    if ((phys->flags & BFPN_FLAG_STREAMING_FULL) && (phys->flags & BFPN_FLAG_LITE_MEMORY))
        return fail(nullptr, BFPN_INVALID_ARG, "--lite-memory and --streaming-full are mutually exclusive");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(nullptr, BFPN_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(nullptr, BFPN_INVALID_ARG, "device ordinal out of range");

    auto* c = new bfpn_ctx();
    c->g = *grid;
    c->ooc = (phys->flags & BFPN_FLAG_STREAMING_FULL) != 0;
    c->p = *phys;
    c->prec = precision;
    c->device = device;
    c->elem = precision == BFPN_PREC_FP64 ? sizeof(double) : sizeof(float);
    c->d = compute_deltas(*grid);
    c->Ng = grid->Ng;
    c->Ny = grid->Ny;
    c->Nz = grid->Nz;
    c->Nmu = grid->Nmu;
    c->Nom = grid->Nom;
    c->nyz = (grid->Ny + 1) * (grid->Nz + 1);
    c->NA = grid->Nmu * grid->Nom;
    c->per_e = static_cast<long long>(c->nyz) * c->NA;
    c->cells = c->per_e * c->Ng;
    auto bail = [&](bfpn_status s) {
        g_create_error = c->err;
        free_all(c);
        if (c->stream) cudaStreamDestroy(c->stream);
        if (c->ev0) cudaEventDestroy(c->ev0);
        if (c->ev1) cudaEventDestroy(c->ev1);
        delete c;
        return s;
    };
    if (set_device(c) != BFPN_OK) return bail(BFPN_CUDA_ERROR);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
        c->err = "stream/event creation failed";
        return bail(BFPN_CUDA_ERROR);
    }
    {
        size_t free_b = 0, total_b = 0;
        if (!c->ooc && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
            const uint64_t need = footprint(*grid, precision, (phys->flags & BFPN_FLAG_LITE_MEMORY) != 0);
            if (need > free_b) {
                char msg[256];
                std::snprintf(msg, sizeof msg,
                              "grid needs about %.2f GiB of device memory but only %.2f GiB is free", need / 1073741824.0,
                              free_b / 1073741824.0);
                c->err = msg;
                return bail(BFPN_OOM);
            }
        }
    }
    choose_transport(c);
    choose_plane_transport(c);
    {
        const size_t per_slice = 2 * static_cast<size_t>(c->NA) * c->elem;
        c->ang_slices = static_cast<int>(std::max<size_t>(1, std::min<size_t>(32, (48 * 1024) / per_slice)));
    }
    const size_t arr = static_cast<size_t>(c->cells) * c->elem;
    const Layout L = layout_of(*grid, precision, c->energy_block);
    c->n_part = L.part_blocks;
    c->hist_cap = L.hist_cap;
    bfpn_status s;
    void* v = nullptr;
#define ALLOC(dst, bytes)                                      \
    if ((s = dalloc(c, &v, (bytes))) != BFPN_OK) return bail(s); \
    dst = static_cast<std::remove_reference_t<decltype(dst)>>(v);
    c->lite = (phys->flags & BFPN_FLAG_LITE_MEMORY) != 0;
    for (int sp = 0; sp < 2; ++sp)
        for (int cf = 0; cf < 2; ++cf) {
            if (c->ooc) {
                void* h = nullptr;
                if (cudaHostAlloc(&h, arr, cudaHostAllocDefault) != cudaSuccess) {
                    cudaGetLastError();
                    c->err = "cannot allocate the pinned host state (" + std::to_string(arr) + " bytes per array)";
                    return bail(BFPN_OOM);
                }
                c->host_allocs.push_back(h);
                c->st[sp][cf] = h;
            } else if (!c->lite || (sp == 0 && cf == 0)) {
                ALLOC(c->st[sp][cf], arr);
            }
        }
    if (!c->tr_inplace && !c->lite && !c->ooc) { ALLOC(c->tmp, arr); }
    const bool need_secondary = !c->lite && !(phys->flags & (BFPN_FLAG_PRIMARY_ONLY | BFPN_FLAG_ENERGY_ONLY));
    if (need_secondary && !c->ooc) {
        ALLOC(c->src, arr);
        // A1 and A2 for the CUDA-core source; the same block holds the
        // tensor-core source's split-bf16 operand
        c->a_bytes = c->prec == BFPN_PREC_MIXED ? std::max(2 * arr, umma_q_bytes(c->per_e, c->Ng)) : 2 * arr;
        ALLOC(c->A1, c->a_bytes);
        c->A2 = static_cast<char*>(c->A1) + arr;
    } else {
        ALLOC(c->src, c->elem);
    }
    ALLOC(c->ecoef_half, static_cast<size_t>(c->Ng) * kEnergyCoef * sizeof(double));
    ALLOC(c->ecoef_op, static_cast<size_t>(c->Ng) * kEnergyCoef * sizeof(double));
    ALLOC(c->dose_coef, 2 * static_cast<size_t>(c->Ng) * sizeof(double));
    ALLOC(c->omega, 2 * static_cast<size_t>(c->NA) * c->elem);
    ALLOC(c->fac_step, static_cast<size_t>(c->Ng) * c->NA * c->elem);
    ALLOC(c->fac_op, static_cast<size_t>(c->Ng) * c->NA * c->elem);
    ALLOC(c->sine_u, static_cast<size_t>(c->Nom) * c->Nom * c->elem);
    ALLOC(c->sine_v, static_cast<size_t>(c->Nmu) * c->Nmu * c->elem);
    if (need_secondary) {
        ALLOC(c->ker_v, static_cast<size_t>(c->Ng) * c->NA * c->NA * c->elem);
    }
    ALLOC(c->e1, static_cast<size_t>(c->Ng) * c->Ng * sizeof(double));
    ALLOC(c->e2, static_cast<size_t>(c->Ng) * c->Ng * sizeof(double));
    ALLOC(c->groups, static_cast<size_t>(c->Ng) * sizeof(int));
    ALLOC(c->gmap, static_cast<size_t>(c->Ng) * sizeof(int));
    ALLOC(c->tile_lo, static_cast<size_t>(c->Ng) * sizeof(int));
    ALLOC(c->tile_hi, static_cast<size_t>(c->Ng) * sizeof(int));
    ALLOC(c->beam_yza, static_cast<size_t>(c->per_e) * sizeof(double));
    ALLOC(c->beam_e, static_cast<size_t>(c->Ng) * sizeof(double));
    // [primary, even steps | secondary | primary, odd steps] x n_part x 2
    ALLOC(c->partials, 6 * static_cast<size_t>(c->n_part) * sizeof(double));
    ALLOC(c->hist_idd, static_cast<size_t>(c->hist_cap) * sizeof(double));
    ALLOC(c->hist_proxy, static_cast<size_t>(c->hist_cap) * sizeof(double));
    ALLOC(c->counter, sizeof(int));
    ALLOC(c->zero_counter, sizeof(int));
    ALLOC(c->dev_err, sizeof(int));
    ALLOC(c->scalar_out, 2 * sizeof(double));
    ALLOC(c->moments, 2 * static_cast<size_t>(c->Ng) * sizeof(double));
    ALLOC(c->plane, static_cast<size_t>(c->nyz) * sizeof(double));
    ALLOC(c->lite_coef, 2 * static_cast<size_t>(c->Ng) * sizeof(double));
#undef ALLOC
    if (need_secondary && !c->ooc) {
        if (cudaMemsetAsync(c->A1, 0, c->a_bytes, c->stream) != cudaSuccess ||
            cudaMemsetAsync(c->src, 0, arr, c->stream) != cudaSuccess) {
            c->err = "memset failed";
            return bail(BFPN_CUDA_ERROR);
        }
    }
    if (cudaMemsetAsync(c->counter, 0, sizeof(int), c->stream) != cudaSuccess ||
        cudaMemsetAsync(c->zero_counter, 0, sizeof(int), c->stream) != cudaSuccess ||
        cudaMemsetAsync(c->dev_err, 0, sizeof(int), c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess) {
        c->err = "memset failed";
        return bail(BFPN_CUDA_ERROR);
    }
    *out = c;
    return BFPN_OK;
}

bfpn_status bfpn_destroy(bfpn_ctx* ctx) {
    if (!ctx) return BFPN_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    free_all(ctx);
    for (cudaStream_t st : {ctx->s_in, ctx->s_out})
        if (st) cudaStreamDestroy(st);
    for (int k = 0; k < 2; ++k)
        for (cudaEvent_t ev : {ctx->ev_in[k], ctx->ev_comp[k], ctx->ev_out[k]})
            if (ev) cudaEventDestroy(ev);
    if (ctx->ev_pass) cudaEventDestroy(ctx->ev_pass);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    delete ctx;
    return BFPN_OK;
}

bfpn_status bfpn_load_tables(bfpn_ctx* c, const double* mu, int32_t mu_rows, const double* sigma_c,
                             int32_t sigma_rows) {
    if (!c) return BFPN_INVALID_ARG;
    if ((!mu && mu_rows > 0) || !sigma_c) return fail(c, BFPN_INVALID_ARG, "null table pointer");
    bfpn_status s = set_device(c);
    if (s != BFPN_OK) return s;
    std::string err;
    BeamTables t;
    // a float-state context keeps only the float angular kernel on the host
    const bool f32_kernel = c->prec == BFPN_PREC_MIXED;
    if (!build_tables(c->g, c->p, mu, mu_rows, sigma_c, sigma_rows, t, err, f32_kernel))
        return fail(c, BFPN_INVALID_ARG, err);
    c->tables = std::move(t);
    c->raw_sigma.assign(sigma_c, sigma_c + std::min<int>(sigma_rows, c->Ng));
    BeamTables& T = c->tables;
    const auto ecoef = energy_coefficients(T, c->p, 0.5 * c->d.dt);
    if ((s = upload_f64(c, c->ecoef_half, ecoef.data(), ecoef.size() * sizeof(double))) != BFPN_OK) return s;
    const auto dose = dose_coefficients(T, c->p);
    if ((s = upload_f64(c, c->dose_coef, dose.data(), dose.size() * sizeof(double))) != BFPN_OK) return s;
    const auto lite = lite_coefficients(T, c->d.dt);
    if ((s = upload_f64(c, c->lite_coef, lite.data(), lite.size() * sizeof(double))) != BFPN_OK) return s;
    if ((s = upload_state_table(c, c->omega, T.omega)) != BFPN_OK) return s;
    c->tr_pairs_ok = transport_pairs_ok(T.omega.data(), c->NA);
    if ((s = upload_state_table(c, c->fac_step, angle_factor(T, c->p, c->d.dt))) != BFPN_OK) return s;
    if ((s = upload_state_table(c, c->sine_u, T.sine_u)) != BFPN_OK) return s;
    if ((s = upload_state_table(c, c->sine_v, T.sine_v)) != BFPN_OK) return s;
    if (c->ker_v) {
        if (f32_kernel) {
            CUDA_TRY(c, cudaMemcpyAsync(c->ker_v, T.ker_v_f.data(), T.ker_v_f.size() * sizeof(float),
                                        cudaMemcpyHostToDevice, c->stream));
            CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        } else if ((s = upload_state_table(c, c->ker_v, T.ker_v)) != BFPN_OK) {
            return s;
        }
    }
    if ((s = upload_f64(c, c->e1, T.ker_e1.data(), T.ker_e1.size() * sizeof(double))) != BFPN_OK) return s;
    if ((s = upload_f64(c, c->e2, T.ker_e2.data(), T.ker_e2.size() * sizeof(double))) != BFPN_OK) return s;
    // source groups that some output band uses and that carry a kernel
    std::vector<char> used(c->Ng, 0);
    for (int e = 0; e < c->Ng; ++e)
        for (int sg = T.band_begin[e]; sg < T.band_end[e]; ++sg) used[sg] = 1;
    std::vector<int> groups;
    for (int sg = 0; sg < c->Ng - 1; ++sg)
        if (used[sg] && T.mu[sg * 3] != 0.0 && T.mu[sg * 3 + 1] != 0.0) groups.push_back(sg);
    c->n_groups = static_cast<int>(groups.size());
    if (!groups.empty() && (s = upload_f64(c, c->groups, groups.data(), groups.size() * sizeof(int))) != BFPN_OK)
        return s;
    {
        std::vector<int> gmap(c->Ng, -1);
        for (size_t k = 0; k < groups.size(); ++k) gmap[groups[k]] = static_cast<int>(k);
        if ((s = upload_f64(c, c->gmap, gmap.data(), gmap.size() * sizeof(int))) != BFPN_OK) return s;
    }
    // tables of an earlier load (a context reused for another beam): the step
    // graph captured their addresses, so it goes too
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    drop_graphs(c);
    dfree(c, c->ablob);
    dfree(c, c->bblob);
    dfree(c, c->eblob);
    { void* w = c->ulist; dfree(c, w); c->ulist = nullptr; }
    { void* w = c->ubegin; dfree(c, w); c->ubegin = nullptr; }
    { void* w = c->ework; dfree(c, w); c->ework = nullptr; }
    { void* w = c->ework_begin; dfree(c, w); c->ework_begin = nullptr; }
    // rows of groups without an angular kernel are read as zeros; an earlier
    // beam's tables may have had a kernel there
    if (c->A1) CUDA_TRY(c, cudaMemsetAsync(c->A1, 0, c->a_bytes, c->stream));
    c->ooc_ready = false;  // the chunk buffers depend on the source groups
    if (c->prec == BFPN_PREC_MIXED && (c->A1 || (c->ooc && c->ker_v)) && !groups.empty()) {
        // tensor-core source: output tiles of <= 256 columns, multiples of 16
        c->umma_ntiles = (c->NA + 255) / 256;
        c->umma_nt = ((c->NA + c->umma_ntiles - 1) / c->umma_ntiles + 15) / 16 * 16;
        // the packed split-bf16 copy of the A operand; without room for it the
        // source's angular stage stays on the fp32 CUDA-core kernel
        const size_t pack = umma_pack_bytes(c->n_groups, c->nyz, c->NA, c->umma_bk);
        size_t free_b = 0, total_b = 0;
        if (!c->ooc && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && pack + (256u << 20) < free_b) {
            void* ab = nullptr;
            if (dalloc(c, &ab, pack) == BFPN_OK) {
                c->ablob = ab;
                // the fused energy kernel writes only real (position, angle)
                // entries; the padding of partial tiles must read as zeros
                CUDA_TRY(c, cudaMemsetAsync(ab, 0, pack, c->stream));
            }
        }
        // B tiles from the float ker_v already on the device
        void* d = nullptr;
        if ((s = dalloc(c, &d, umma_blob_bytes(c->n_groups, c->NA, c->umma_nt, c->umma_bk))) != BFPN_OK) return s;
        c->bblob = d;
        CUDA_TRY(c, launch_build_umma_blob(as<const float>(c->ker_v), c->groups, c->n_groups, c->NA, c->umma_nt,
                                           c->umma_bk, static_cast<uint8_t*>(d), c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        // the kernel blocks' non-zero k chunks and column ranges (the kernel is
        // sparse: entries below the threshold were dropped)
        if (!T.ker_v_f.empty()) {
            std::vector<int4> ul;
            std::vector<int> ub;
            build_umma_ranges(T.ker_v_f.data(), groups.data(), c->n_groups, c->NA, c->umma_nt, c->umma_bk,
                              c->umma_ntiles, ul, ub);
            void *dl = nullptr, *dbg = nullptr;
            if ((s = dalloc(c, &dl, std::max<size_t>(16, ul.size() * sizeof(int4)))) != BFPN_OK) return s;
            c->ulist = static_cast<int4*>(dl);
            if (!ul.empty() && (s = upload_f64(c, dl, ul.data(), ul.size() * sizeof(int4))) != BFPN_OK) return s;
            if ((s = dalloc(c, &dbg, ub.size() * sizeof(int))) != BFPN_OK) return s;
            c->ubegin = static_cast<int*>(dbg);
            if ((s = upload_f64(c, dbg, ub.data(), ub.size() * sizeof(int))) != BFPN_OK) return s;
            CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        }
        // energy stage: banded coefficient tiles and per-output-tile work lists
        std::vector<uint8_t> eb;
        std::vector<int> work, begin;
        build_energy_umma(T.ker_e1.data(), T.ker_e2.data(), T.band_begin.data(), T.band_end.data(), c->Ng, c->d.dg,
                          eb, work, begin, c->e_emax);
        c->e_et = static_cast<int>(begin.size()) - 1;
        void *de = nullptr, *dw = nullptr, *db = nullptr;
        if ((s = dalloc(c, &de, eb.size())) != BFPN_OK) return s;
        c->eblob = de;
        if ((s = upload_f64(c, de, eb.data(), eb.size())) != BFPN_OK) return s;
        if ((s = dalloc(c, &dw, std::max<size_t>(16, work.size() * sizeof(int)))) != BFPN_OK) return s;
        c->ework = static_cast<int*>(dw);
        if (!work.empty() && (s = upload_f64(c, dw, work.data(), work.size() * sizeof(int))) != BFPN_OK) return s;
        if ((s = dalloc(c, &db, begin.size() * sizeof(int))) != BFPN_OK) return s;
        c->ework_begin = static_cast<int*>(db);
        if ((s = upload_f64(c, db, begin.data(), begin.size() * sizeof(int))) != BFPN_OK) return s;
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    }
    const int tiles = (c->Ng + c->tile_e - 1) / c->tile_e;
    std::vector<int> lo(tiles, 0), hi(tiles, 0);
    for (int tI = 0; tI < tiles; ++tI) {
        int l = c->Ng, h = 0;
        for (int e = tI * c->tile_e; e < std::min(c->Ng, (tI + 1) * c->tile_e); ++e)
            if (T.band_end[e] > T.band_begin[e]) {
                l = std::min(l, T.band_begin[e]);
                h = std::max(h, T.band_end[e]);
            }
        if (l < h) {
            lo[tI] = l;
            hi[tI] = h;
        }
    }
    if ((s = upload_f64(c, c->tile_lo, lo.data(), lo.size() * sizeof(int))) != BFPN_OK) return s;
    if ((s = upload_f64(c, c->tile_hi, hi.data(), hi.size() * sizeof(int))) != BFPN_OK) return s;
    if ((s = upload_f64(c, c->beam_yza, T.beam_yza.data(), T.beam_yza.size() * sizeof(double))) != BFPN_OK) return s;
    if ((s = upload_f64(c, c->beam_e, T.beam_e.data(), T.beam_e.size() * sizeof(double))) != BFPN_OK) return s;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->tables_loaded = true;
    c->ecoef_op_dt = -1.0;
    c->fac_op_dt = -1.0;
    return BFPN_OK;
}

bfpn_status bfpn_init_beam(bfpn_ctx* c) {
    if (!c) return BFPN_INVALID_ARG;
    if (!c->tables_loaded) return fail(c, BFPN_NOT_READY, "tables not loaded (bfpn_load_tables)");
    bfpn_status s = set_device(c);
    if (s != BFPN_OK) return s;
    const size_t arr = static_cast<size_t>(c->cells) * c->elem;
    if (c->ooc) {  // group chunk by group chunk into the host array
        if ((s = ensure_ooc(c)) != BFPN_OK) return s;
        const size_t row = static_cast<size_t>(c->per_e) * c->elem;
        for (int e0 = 0; e0 < c->Ng; e0 += c->ecg) {
            const int g = std::min(c->ecg, c->Ng - e0);
            if (c->prec == BFPN_PREC_FP64)
                CUDA_TRY(c, launch_init_beam<double>(as<double>(c->dgc[0]), c->beam_yza, c->beam_e + e0, c->per_e, g,
                                                     c->stream));
            else
                CUDA_TRY(c, launch_init_beam<float>(as<float>(c->dgc[0]), c->beam_yza, c->beam_e + e0, c->per_e, g,
                                                    c->stream));
            CUDA_TRY(c, cudaMemcpyAsync(static_cast<char*>(c->st[0][0]) + e0 * row, c->dgc[0], g * row,
                                        cudaMemcpyDeviceToHost, c->stream));
        }
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        for (void* X : {c->st[0][1], c->st[1][0], c->st[1][1]}) std::memset(X, 0, arr);
        CUDA_TRY(c, cudaMemsetAsync(c->counter, 0, sizeof(int), c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        c->beam_ready = true;
        c->steps_done = 0;
        c->secondary_zero = true;
        return BFPN_OK;
    }
    if (c->prec == BFPN_PREC_FP64) {
        CUDA_TRY(c, launch_init_beam<double>(as<double>(c->st[0][0]), c->beam_yza, c->beam_e, c->per_e, c->Ng, c->stream));
    } else {
        CUDA_TRY(c, launch_init_beam<float>(as<float>(c->st[0][0]), c->beam_yza, c->beam_e, c->per_e, c->Ng, c->stream));
    }
    for (void* X : {c->st[0][1], c->st[1][0], c->st[1][1]})
        if (X) CUDA_TRY(c, cudaMemsetAsync(X, 0, arr, c->stream));
    CUDA_TRY(c, cudaMemsetAsync(c->counter, 0, sizeof(int), c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->beam_ready = true;
    c->steps_done = 0;
    c->secondary_zero = true;
    return BFPN_OK;
}

bfpn_status bfpn_step_async(bfpn_ctx* c, int32_t nsteps) {
    if (!c) return BFPN_INVALID_ARG;
    bfpn_status s = set_device(c);
    if (s != BFPN_OK) return s;
    return run_steps(c, nsteps);
}

bfpn_status bfpn_sync(bfpn_ctx* c) {
    if (!c) return BFPN_INVALID_ARG;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    CUDA_TRY(c, collect_profile(c));
    return check_device_error(c);
}

bfpn_status bfpn_history_download(bfpn_ctx* c, int32_t first, int32_t count, double* idd_out, double* proxy_out) {
    if (!c) return BFPN_INVALID_ARG;
    if (first < 0 || count < 0 || first + count > c->steps_done)
        return fail(c, BFPN_INVALID_ARG, "history range outside the steps done");
    if (count == 0) return BFPN_OK;
    if (idd_out)
        CUDA_TRY(c, cudaMemcpyAsync(idd_out, c->hist_idd + first, count * sizeof(double), cudaMemcpyDeviceToHost,
                                    c->stream));
    if (proxy_out)
        CUDA_TRY(c, cudaMemcpyAsync(proxy_out, c->hist_proxy + first, count * sizeof(double), cudaMemcpyDeviceToHost,
                                    c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return BFPN_OK;
}

bfpn_status bfpn_step(bfpn_ctx* c, int32_t nsteps, double* idd_out, double* proxy_out) {
    if (!c) return BFPN_INVALID_ARG;
    const int first = c->steps_done;
    bfpn_status s = bfpn_step_async(c, nsteps);
    if (s != BFPN_OK) return s;
    if (idd_out || proxy_out) {
        s = bfpn_history_download(c, first, nsteps, idd_out, proxy_out);
        if (s != BFPN_OK) return s;
    }
    return bfpn_sync(c);
}

int32_t bfpn_steps_done(const bfpn_ctx* c) { return c ? c->steps_done : -1; }

uint64_t bfpn_cells(const bfpn_ctx* c) { return c ? static_cast<uint64_t>(c->cells) : 0; }

void* bfpn_stream(bfpn_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

bfpn_status bfpn_energy_eq15(bfpn_ctx* c, int32_t species, double dt, int32_t with_source) {
    if (!c) return BFPN_INVALID_ARG;
    if (c->ooc) return fail(c, BFPN_INVALID_ARG, "needs a device-resident state (not available in the out-of-core mode)");
    if (!c->tables_loaded) return fail(c, BFPN_NOT_READY, "tables not loaded");
    if (species < 0 || species > 1 || !(dt > 0)) return fail(c, BFPN_INVALID_ARG, "bad species or dt");
    if (c->lite) return fail(c, BFPN_INVALID_ARG, "not available in lite-memory mode (psi^1 of the primary only)");
    if (with_source && (species != 1 || !c->A1))
        return fail(c, BFPN_INVALID_ARG, "the source applies to the secondary species of a context that has one");
    bfpn_status s = set_device(c);
    if (s != BFPN_OK) return s;
    if (dt != c->ecoef_op_dt) {
        const auto k = energy_coefficients(c->tables, c->p, dt);
        if ((s = upload_f64(c, c->ecoef_op, k.data(), k.size() * sizeof(double))) != BFPN_OK) return s;
        c->ecoef_op_dt = dt;
    }
    if (c->prec == BFPN_PREC_FP64) CUDA_TRY(c, enq_energy<double>(c, species, c->ecoef_op, with_source != 0, nullptr));
    else CUDA_TRY(c, enq_energy<float>(c, species, c->ecoef_op, with_source != 0, nullptr));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return check_device_error(c);
}

bfpn_status bfpn_transport_eq18(bfpn_ctx* c, int32_t species, int32_t coef, double dt, int32_t preserve_sign) {
    if (!c) return BFPN_INVALID_ARG;
    if (c->ooc) return fail(c, BFPN_INVALID_ARG, "needs a device-resident state (not available in the out-of-core mode)");
    if (!c->tables_loaded) return fail(c, BFPN_NOT_READY, "tables not loaded");
    if (species < 0 || species > 1 || coef < 0 || coef > 1 || !(dt > 0))
        return fail(c, BFPN_INVALID_ARG, "bad species, coef or dt");
    if (c->lite) return fail(c, BFPN_INVALID_ARG, "not available in lite-memory mode (psi^1 of the primary only)");
    bfpn_status s = set_device(c);
    if (s != BFPN_OK) return s;
    void* X = c->st[species][coef];
    void* Y = transport_in_place(c) ? X : c->tmp;
    if (c->prec == BFPN_PREC_FP64) CUDA_TRY(c, enq_transport<double>(c, X, Y, dt, preserve_sign != 0));
    else CUDA_TRY(c, enq_transport<float>(c, X, Y, dt, preserve_sign != 0));
    if (Y != X)
        CUDA_TRY(c, cudaMemcpyAsync(X, Y, static_cast<size_t>(c->cells) * c->elem, cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return BFPN_OK;
}

bfpn_status bfpn_angle_eq19(bfpn_ctx* c, int32_t species, int32_t coef, double dt) {
    if (!c) return BFPN_INVALID_ARG;
    if (c->ooc) return fail(c, BFPN_INVALID_ARG, "needs a device-resident state (not available in the out-of-core mode)");
    if (!c->tables_loaded) return fail(c, BFPN_NOT_READY, "tables not loaded");
    if (species < 0 || species > 1 || coef < 0 || coef > 1 || !(dt > 0))
        return fail(c, BFPN_INVALID_ARG, "bad species, coef or dt");
    if (c->lite) return fail(c, BFPN_INVALID_ARG, "not available in lite-memory mode (psi^1 of the primary only)");
    bfpn_status s = set_device(c);
    if (s != BFPN_OK) return s;
    if (dt != c->fac_op_dt) {
        if ((s = upload_state_table(c, c->fac_op, angle_factor(c->tables, c->p, dt))) != BFPN_OK) return s;
        c->fac_op_dt = dt;
    }
    if (c->prec == BFPN_PREC_FP64) CUDA_TRY(c, enq_angle<double>(c, c->st[species][coef], c->fac_op));
    else CUDA_TRY(c, enq_angle<float>(c, c->st[species][coef], c->fac_op));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return BFPN_OK;
}

bfpn_status bfpn_secondary_source(bfpn_ctx* c) {
    if (!c) return BFPN_INVALID_ARG;
    if (c->ooc) return fail(c, BFPN_INVALID_ARG, "needs a device-resident state (not available in the out-of-core mode)");
    if (!c->tables_loaded) return fail(c, BFPN_NOT_READY, "tables not loaded");
    if (!c->A1) return fail(c, BFPN_INVALID_ARG, "context has no secondary species (primary-only or energy-only)");
    bfpn_status s = set_device(c);
    if (s != BFPN_OK) return s;
    if (c->prec == BFPN_PREC_FP64) CUDA_TRY(c, enq_source<double>(c));
    else CUDA_TRY(c, enq_source<float>(c));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return check_device_error(c);
}

bfpn_status bfpn_set_option(bfpn_ctx* c, int32_t option, int32_t value) {
    if (!c) return BFPN_INVALID_ARG;
    switch (option) {
        case BFPN_OPT_TENSOR_CORES:
            if (c->use_umma != (value != 0) && c->A1) {
                // the two source paths keep different layouts in the A block,
                // and both read the rows the other path wrote as zeros
                CUDA_TRY(c, cudaMemsetAsync(c->A1, 0, c->a_bytes, c->stream));
                CUDA_TRY(c, cudaStreamSynchronize(c->stream));
            }
            c->use_umma = value != 0;
            break;
        case BFPN_OPT_CUDA_GRAPHS:
            c->use_graphs = value != 0 && !c->profiling;
            break;
        case BFPN_OPT_STEP_OVERLAP:
            if (value < 0 || value > 2) return fail(c, BFPN_INVALID_ARG, "step overlap: 0, 1 or 2");
            c->overlap = value != 0;
            c->split_chains = value == 2;
            break;
        case BFPN_OPT_PAIRED_ANGLES:
            c->tr_pairs = value != 0;
            break;
        case BFPN_OPT_LANE_CHUNK:
        case BFPN_OPT_ENERGY_CHUNK:
            if (value < 1) return fail(c, BFPN_INVALID_ARG, "chunk sizes must be positive");
            (option == BFPN_OPT_LANE_CHUNK ? c->ooc_lane_req : c->ooc_group_req) = value;
            break;
        case BFPN_OPT_FUSED_ENERGY:
            c->fuse_energy = value != 0;
            break;
        case BFPN_OPT_STREAM_TRANSPORT:
            if (value < 0 || value > 2) return fail(c, BFPN_INVALID_ARG, "stream transport: 0, 1 or 2");
            if (value == 2 && !c->tr_stream_ok)
                return fail(c, BFPN_INVALID_ARG, "no row-streaming transport for this plane size / precision");
            c->tr_stream = value;
            break;
        case BFPN_OPT_CLUSTER_TRANSPORT:
            if (value < 0 || value > 2) return fail(c, BFPN_INVALID_ARG, "cluster transport: 0, 1 or 2");
            if (value == 2 && !c->tr_cluster_ok)
                return fail(c, BFPN_INVALID_ARG, "no cluster transport kernel for this plane size / precision");
            c->tr_cluster = value;
            break;
        case BFPN_OPT_PLANE_TRANSPORT: {
            const bool f32 = c->elem == 4;
            if (value != 0 && !c->tr_plane_ok && !c->tr_tile_ok)
                return fail(c, BFPN_INVALID_ARG, "no unrolled transport kernel for this plane size");
            if (value > 1) {
                const bool ok = c->tr_plane_ok ? (f32 ? (value == 8 || value == 16) : (value == 4 || value == 8))
                                               : (f32 ? (value == 4 || value == 8) : (value == 2 || value == 4));
                if (!ok)
                    return fail(c, BFPN_INVALID_ARG,
                                "angle chunk: 8/16 (float) or 4/8 (double) for whole planes, 4/8 (float) or 2/4 "
                                "(double) for tiled planes");
                if (c->tr_plane_ok && transport_plane_smem(c->Ny + 1, value, c->elem) > 200 * 1024)
                    return fail(c, BFPN_INVALID_ARG, "plane transport chunk needs too much shared memory");
            }
            if (value != 0 && value != 1 && !(value > 1)) return fail(c, BFPN_INVALID_ARG, "bad option value");
            if (c->tr_plane_ok) {
                c->tr_plane = value != 0;
                if (value > 1) c->tr_plane_ac = value;
            } else {
                c->tr_tile = value != 0;
                if (value > 1) c->tr_tile_ac = value;
            }
            break;
        }
        default:
            return fail(c, BFPN_INVALID_ARG, "unknown option");
    }
    drop_graphs(c);
    return BFPN_OK;
}

bfpn_status bfpn_idd(bfpn_ctx* c, double* idd, double* proxy) {
    if (!c) return BFPN_INVALID_ARG;
    if (c->ooc) return fail(c, BFPN_INVALID_ARG, "needs a device-resident state (not available in the out-of-core mode)");
    if (!c->tables_loaded) return fail(c, BFPN_NOT_READY, "tables not loaded");
    bfpn_status s = set_device(c);
    if (s != BFPN_OK) return s;
    const int n = idd_partials_grid(c->per_e);
    if (c->lite) {  // computeIntegratedDepthDoseLite (bfpm_solver.cu:3528-3558): psi^1 only, proxy 0
        const int trap = (c->p.flags & BFPN_FLAG_TRAPEZOIDAL_YZ) ? 1 : 0;
        if (c->prec == BFPN_PREC_FP64)
            CUDA_TRY(c, launch_idd_partials<double>(as<double>(c->st[0][0]), nullptr, c->dose_coef, c->Ng, c->per_e,
                                                    c->NA, c->Ny, c->Nz, trap, 0, c->partials, n, c->stream));
        else
            CUDA_TRY(c, launch_idd_partials<float>(as<float>(c->st[0][0]), nullptr, c->dose_coef, c->Ng, c->per_e,
                                                   c->NA, c->Ny, c->Nz, trap, 0, c->partials, n, c->stream));
        const double w = c->d.du * c->d.dv * c->d.dy * c->d.dz;
        CUDA_TRY(c, launch_finalize_idd(c->partials, n, nullptr, 0, w, c->d.dg, c->scalar_out, c->scalar_out + 1,
                                        c->zero_counter, 1, 0, c->stream));
        double h[2] = {0, 0};
        CUDA_TRY(c, cudaMemcpyAsync(h, c->scalar_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        if (idd) *idd = h[0];
        if (proxy) *proxy = h[1];
        return BFPN_OK;
    }
    const int trap = (c->p.flags & BFPN_FLAG_TRAPEZOIDAL_YZ) ? 1 : 0;
    double* pP = c->partials;
    double* pS = c->partials + 2 * c->n_part;
    if (c->prec == BFPN_PREC_FP64) {
        CUDA_TRY(c, launch_idd_partials<double>(as<double>(c->st[0][0]), as<double>(c->st[0][1]), c->dose_coef, c->Ng,
                                                c->per_e, c->NA, c->Ny, c->Nz, trap, 1, pP, n, c->stream));
        CUDA_TRY(c, launch_idd_partials<double>(as<double>(c->st[1][0]), as<double>(c->st[1][1]), c->dose_coef, c->Ng,
                                                c->per_e, c->NA, c->Ny, c->Nz, trap, 0, pS, n, c->stream));
    } else {
        CUDA_TRY(c, launch_idd_partials<float>(as<float>(c->st[0][0]), as<float>(c->st[0][1]), c->dose_coef, c->Ng,
                                               c->per_e, c->NA, c->Ny, c->Nz, trap, 1, pP, n, c->stream));
        CUDA_TRY(c, launch_idd_partials<float>(as<float>(c->st[1][0]), as<float>(c->st[1][1]), c->dose_coef, c->Ng,
                                               c->per_e, c->NA, c->Ny, c->Nz, trap, 0, pS, n, c->stream));
    }
    const double w = c->d.du * c->d.dv * c->d.dy * c->d.dz;
    CUDA_TRY(c, launch_finalize_idd(pP, n, pS, n, w, c->d.dg, c->scalar_out, c->scalar_out + 1, c->zero_counter, 1, 0,
                                    c->stream));
    double h[2] = {0, 0};
    CUDA_TRY(c, cudaMemcpyAsync(h, c->scalar_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (idd) *idd = h[0];
    if (proxy) *proxy = h[1];
    return BFPN_OK;
}

bfpn_status bfpn_state_upload(bfpn_ctx* c, int32_t species, int32_t coef, const double* host) {
    if (!c || !host) return BFPN_INVALID_ARG;
    if (species < 0 || species > 1 || coef < 0 || coef > 1) return fail(c, BFPN_INVALID_ARG, "bad species or coef");
    if (!c->st[species][coef])
        return fail(c, BFPN_INVALID_ARG, "lite-memory mode holds only psi^1 of the primary (species 0, coef 0)");
    bfpn_status s = set_device(c);
    if (s != BFPN_OK) return s;
    if (c->ooc) {  // the state is host memory: convert in place
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        if (c->prec == BFPN_PREC_FP64) std::memcpy(c->st[species][coef], host, c->cells * sizeof(double));
        else {
            float* d = static_cast<float*>(c->st[species][coef]);
            for (long long i = 0; i < c->cells; ++i) d[i] = static_cast<float>(host[i]);
        }
    } else {
        s = c->prec == BFPN_PREC_FP64 ? upload_as<double>(c, c->st[species][coef], host, c->cells)
                                      : upload_as<float>(c, c->st[species][coef], host, c->cells);
    }
    if (s != BFPN_OK) return s;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (species == 1) c->secondary_zero = false;
    c->beam_ready = true;
    return BFPN_OK;
}

bfpn_status bfpn_state_download(bfpn_ctx* c, int32_t species, int32_t coef, double* host) {
    if (!c || !host) return BFPN_INVALID_ARG;
    if (species < 0 || species > 1 || coef < 0 || coef > 1) return fail(c, BFPN_INVALID_ARG, "bad species or coef");
    if (!c->st[species][coef])
        return fail(c, BFPN_INVALID_ARG, "lite-memory mode holds only psi^1 of the primary (species 0, coef 0)");
    bfpn_status s = set_device(c);
    if (s != BFPN_OK) return s;
    if (c->ooc) {
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        if (c->prec == BFPN_PREC_FP64) std::memcpy(host, c->st[species][coef], c->cells * sizeof(double));
        else {
            const float* d = static_cast<const float*>(c->st[species][coef]);
            for (long long i = 0; i < c->cells; ++i) host[i] = static_cast<double>(d[i]);
        }
        return BFPN_OK;
    }
    return c->prec == BFPN_PREC_FP64 ? download_as<double>(c, c->st[species][coef], host, c->cells)
                                     : download_as<float>(c, c->st[species][coef], host, c->cells);
}

bfpn_status bfpn_source_download(bfpn_ctx* c, double* host) {
    if (!c || !host) return BFPN_INVALID_ARG;
    if (c->ooc) return fail(c, BFPN_INVALID_ARG, "needs a device-resident state (not available in the out-of-core mode)");
    if (!c->A1) return fail(c, BFPN_INVALID_ARG, "context has no secondary species");
    bfpn_status s = set_device(c);
    if (s != BFPN_OK) return s;
    return c->prec == BFPN_PREC_FP64 ? download_as<double>(c, c->src, host, c->cells)
                                     : download_as<float>(c, c->src, host, c->cells);
}

bfpn_status bfpn_table_download(bfpn_ctx* c, int32_t which, double* host, uint64_t n) {
    if (!c || !host) return BFPN_INVALID_ARG;
    if (!c->tables_loaded) return fail(c, BFPN_NOT_READY, "tables not loaded");
    std::vector<double> tmp;
    if (which == BFPN_TABLE_KER_V) angular_kernel_f64(c->tables);
    const TableView src = table_of(c->tables, which, tmp);
    if (!src.known) return fail(c, BFPN_INVALID_ARG, "unknown table id");
    if (src.size > n) return fail(c, BFPN_INVALID_ARG, "host buffer too small for the table");
    if (src.size) std::memcpy(host, src.data, src.size * sizeof(double));
    return BFPN_OK;
}

bfpn_status bfpn_set_profiling(bfpn_ctx* c, int32_t on) {
    if (!c) return BFPN_INVALID_ARG;
    CUDA_TRY(c, collect_profile(c));
    c->profiling = on != 0;
    c->use_graphs = !c->profiling;
    return BFPN_OK;
}

bfpn_status bfpn_kernel_profile(bfpn_ctx* c, double* ms_out, int32_t* launches_out, int32_t n) {
    if (!c) return BFPN_INVALID_ARG;
    CUDA_TRY(c, collect_profile(c));
    for (int i = 0; i < std::min<int>(n, BFPN_KERNEL_CLASSES); ++i) {
        if (ms_out) ms_out[i] = c->prof_ms[i];
        if (launches_out) launches_out[i] = c->prof_n[i];
    }
    return BFPN_OK;
}

bfpn_status bfpn_kernel_profile_reset(bfpn_ctx* c) {
    if (!c) return BFPN_INVALID_ARG;
    CUDA_TRY(c, collect_profile(c));
    for (int i = 0; i < BFPN_KERNEL_CLASSES; ++i) {
        c->prof_ms[i] = 0.0;
        c->prof_n[i] = 0;
    }
    return BFPN_OK;
}

int32_t bfpn_kernels_per_step(bfpn_ctx* c) { return c ? c->kernels_per_step : -1; }

int32_t bfpn_source_groups(bfpn_ctx* c) { return c ? c->n_groups : -1; }

bfpn_status bfpn_timed_steps(bfpn_ctx* c, int32_t nsteps, double* elapsed_ms) {
    if (!c || !elapsed_ms) return BFPN_INVALID_ARG;
    bfpn_status s = set_device(c);
    if (s != BFPN_OK) return s;
    CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));
    s = run_steps(c, nsteps);
    if (s != BFPN_OK) return s;
    CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
    CUDA_TRY(c, cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    *elapsed_ms = ms;
    CUDA_TRY(c, collect_profile(c));
    return check_device_error(c);
}

bfpn_status bfpn_setup_summary(bfpn_ctx* c, bfpn_setup_info* out) {
    if (!c || !out) return BFPN_INVALID_ARG;
    if (!c->tables_loaded) return fail(c, BFPN_NOT_READY, "tables not loaded");
    const BeamTables& T = c->tables;
    out->mu_rows = T.mu_rows;
    // bfpm_solver.cu:1494-1500
    const int bg = std::max(0, std::min(static_cast<int>((c->p.beam_energy - 1.0) / c->d.dg), c->Ng - 1));
    out->beam_group = bg;
    out->beam_group_energy = (bg + 0.5) * c->d.dg + 1.0;
    out->sigma_fitted = c->raw_sigma.empty() ? 0.0 : c->raw_sigma[bg];
    out->sigma_used = T.sigma[bg];
    out->omega_center_y = T.omega_center_y;
    out->omega_center_z = T.omega_center_z;
    out->spatial_mass = T.spatial_mass;
    out->angular_mass = T.angular_mass;
    out->energy_mass = T.energy_mass;
    out->initial_scale = T.initial_scale;
    return BFPN_OK;
}

bfpn_status bfpn_energy_moments(bfpn_ctx* c, double* out) {
    if (!c || !out) return BFPN_INVALID_ARG;
    if (c->ooc) return fail(c, BFPN_INVALID_ARG, "needs a device-resident state (not available in the out-of-core mode)");
    if (c->lite) return fail(c, BFPN_INVALID_ARG, "not available in lite-memory mode (psi^1 of the primary only)");
    bfpn_status s = set_device(c);
    if (s != BFPN_OK) return s;
    const double w = c->d.du * c->d.dv * c->d.dy * c->d.dz;
    if (c->prec == BFPN_PREC_FP64)
        CUDA_TRY(c, launch_energy_moments<double>(as<double>(c->st[0][0]), as<double>(c->st[0][1]), as<double>(c->st[1][0]),
                                                  as<double>(c->st[1][1]), c->Ng, c->per_e, w, c->moments, c->stream));
    else
        CUDA_TRY(c, launch_energy_moments<float>(as<float>(c->st[0][0]), as<float>(c->st[0][1]), as<float>(c->st[1][0]),
                                                 as<float>(c->st[1][1]), c->Ng, c->per_e, w, c->moments, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(out, c->moments, 2 * static_cast<size_t>(c->Ng) * sizeof(double),
                                cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return BFPN_OK;
}

bfpn_status bfpn_spot_plane(bfpn_ctx* c, double* plane) {
    if (!c || !plane) return BFPN_INVALID_ARG;
    if (c->ooc) return fail(c, BFPN_INVALID_ARG, "needs a device-resident state (not available in the out-of-core mode)");
    if (c->lite) return fail(c, BFPN_INVALID_ARG, "not available in lite-memory mode (psi^1 of the primary only)");
    if (!c->tables_loaded) return fail(c, BFPN_NOT_READY, "tables not loaded");
    bfpn_status s = set_device(c);
    if (s != BFPN_OK) return s;
    const double dudv = c->d.du * c->d.dv;
    if (c->prec == BFPN_PREC_FP64)
        CUDA_TRY(c, launch_spot_plane<double>(as<double>(c->st[0][0]), as<double>(c->st[0][1]), as<double>(c->st[1][0]),
                                              as<double>(c->st[1][1]), c->dose_coef, c->Ng, c->nyz, c->NA, dudv,
                                              c->plane, c->stream));
    else
        CUDA_TRY(c, launch_spot_plane<float>(as<float>(c->st[0][0]), as<float>(c->st[0][1]), as<float>(c->st[1][0]),
                                             as<float>(c->st[1][1]), c->dose_coef, c->Ng, c->nyz, c->NA, dudv,
                                             c->plane, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(plane, c->plane, static_cast<size_t>(c->nyz) * sizeof(double), cudaMemcpyDeviceToHost,
                                c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return BFPN_OK;
}

int32_t bfpn_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

bfpn_status bfpn_device_memory(int32_t device, uint64_t* free_bytes, uint64_t* total_bytes) {
    int n = 0, prev = -1;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return BFPN_NO_DEVICE;
    }
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    size_t f = 0, t = 0;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaMemGetInfo(&f, &t);
    if (prev >= 0) cudaSetDevice(prev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return BFPN_CUDA_ERROR;
    }
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
    return BFPN_OK;
}

int32_t bfpn_device_info(int32_t device, char* buf, int32_t buf_len) {
    cudaDeviceProp prop;
    if (!buf || buf_len <= 0 || cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    int n = std::snprintf(buf, buf_len,
                          "Device %d: %s\n  Compute Capability: %d.%d\n  Total Memory: %zu MB\n"
                          "  Multiprocessors: %d\n  Max Threads/Block: %d\n",
                          device, prop.name, prop.major, prop.minor, prop.totalGlobalMem / (1024 * 1024),
                          prop.multiProcessorCount, prop.maxThreadsPerBlock);
    return n < buf_len ? n : buf_len - 1;
}

}  // extern "C"

// ============================================================================
// Per-slot step pieces for bundles (bundle.cu): the arguments enq_energy,
// enq_transport and enq_angle would build for this context, the source on a
// given stream, and the IDD finalisation.
// ============================================================================
namespace bfpn {

std::string bundle_ready(const bfpn_ctx* c) {
    if (!c) return "null context";
    if (c->prec != BFPN_PREC_MIXED) return "a bundle holds mixed-precision beams";
    if (c->lite || c->ooc) return "lite-memory and out-of-core beams run alone";
    const unsigned fl = c->p.flags;
    if (fl & (BFPN_FLAG_ENERGY_ONLY | BFPN_FLAG_PRIMARY_ONLY | BFPN_FLAG_NO_TRANSPORT | BFPN_FLAG_NO_ANGLE |
              BFPN_FLAG_LEGACY_ENERGY))
        return "a bundle runs the eq15 step with transport, angular diffusion and secondaries";
    if (!c->tables_loaded || !c->beam_ready) return "load the tables and the initial beam first";
    if (!(c->tr_pairs && c->tr_pairs_ok)) return "the angle pairs do not share direction signs";
    if (!(stream_transport(c) || cluster_transport(c) || c->tr_plane))
        return "no whole-plane, row-streaming or cluster transport kernel for this plane";
    if (c->Nom != c->Nmu || c->Nom % 2 != 0 || c->Nom < 4 || c->Nom > 32 || c->Nom == 26 || c->Nom == 30)
        return "the angular grid must be square with an even side in 4..24, 28 or 32";
    if (c->nyz < angle_slots_tile(c->Nom)) return "the plane is smaller than one DST tile";
    if (c->per_e % 4 != 0) return "Ny+1, Nz+1, Nmu, Nom give a lane count that is not a multiple of 4";
    return "";
}

bool bundle_tc_source(const bfpn_ctx* c) {
    return c && (c->n_groups == 0 || (c->use_umma && c->ablob && c->bblob && c->eblob));
}

EnergyArgs<float> bundle_energy_args(bfpn_ctx* c, int species, bool with_source, double* partials) {
    EnergyArgs<float> a;
    a.F = as<float>(c->st[species][0]);
    a.f = as<float>(c->st[species][1]);
    a.src = with_source ? as<const float>(c->src) : nullptr;
    a.coef = c->ecoef_half;
    a.Ng = c->Ng;
    a.lanes = c->per_e;
    a.mode = (c->p.flags & BFPN_FLAG_EQ15_STRAGGLING) ? EMODE_EQ15_STRAG : EMODE_EQ15;
    a.partials = partials;
    a.dose_coef = c->dose_coef;
    a.NA = c->NA;
    a.Ny = c->Ny;
    a.Nz = c->Nz;
    a.trapezoidal = (c->p.flags & BFPN_FLAG_TRAPEZOIDAL_YZ) ? 1 : 0;
    return a;
}

TransportArgs<float> bundle_transport_args(bfpn_ctx* c, int species, int coef, bool preserve_sign) {
    TransportArgs<float> a;
    a.in = as<const float>(c->st[species][coef]);
    a.out = as<float>(c->st[species][coef]);
    a.omega = as<const float>(c->omega);
    a.Ny = c->Ny;
    a.Nz = c->Nz;
    a.NA = c->NA;
    a.Ng = c->Ng;
    a.dt = static_cast<float>(0.5 * c->d.dt);
    a.dy = static_cast<float>(c->d.dy);
    a.dz = static_cast<float>(c->d.dz);
    a.tile_y = c->tr_ty;
    a.tile_z = c->tr_tz;
    a.preserve_sign = preserve_sign ? 1 : 0;
    a.pairs = 1;
    return a;
}

AngleArgs<float> bundle_angle_args(bfpn_ctx* c, int species, int coef, int* err) {
    AngleArgs<float> a;
    a.F = as<float>(c->st[species][coef]);
    a.fac = as<const float>(c->fac_step);
    a.sine_u = as<const float>(c->sine_u);
    a.sine_v = as<const float>(c->sine_v);
    a.Nom = c->Nom;
    a.Nmu = c->Nmu;
    a.nyz = c->nyz;
    a.Ng = c->Ng;
    a.slices_per_block = angle_slots_tile(c->Nom);
    a.err = err;
    a.pairs = 1;
    return a;
}

cudaError_t bundle_source(bfpn_ctx* c, cudaStream_t s) {
    cudaStream_t own = c->stream;
    c->stream = s;
    const cudaError_t e = enq_source<float>(c, nullptr);
    c->stream = own;
    return e;
}

double* bundle_partials(bfpn_ctx* c, int species) {
    return species == 0 ? primary_partials(c, 0) : c->partials + 2 * static_cast<size_t>(c->n_part);
}

IddFinalArgs bundle_finalize_args(bfpn_ctx* c, bool secondary) {
    IddFinalArgs f;
    const int nP = energy_grid(c->per_e, c->energy_block);
    f.p = bundle_partials(c, 0);
    f.n = nP;
    f.p2 = secondary ? bundle_partials(c, 1) : nullptr;
    f.n2 = secondary ? nP : 0;
    f.idd_scale = c->d.du * c->d.dv * c->d.dy * c->d.dz;
    f.proxy_scale = c->d.dg;
    f.hist_idd = c->hist_idd;
    f.hist_proxy = c->hist_proxy;
    f.counter = c->counter;
    f.capacity = c->hist_cap;
    return f;
}

bfpn_status bundle_reserve_history(bfpn_ctx* c, int n) { return ensure_history(c, c->steps_done + n); }

int bundle_cluster_size(const bfpn_ctx* c) { return cluster_transport(c) ? transport_cluster_size(c->Ny + 1) : 0; }

bool bundle_stream_transport(const bfpn_ctx* c) { return stream_transport(c); }

std::string bundle_class_key(const bfpn_ctx* c) {
    char buf[160];
    std::snprintf(buf, sizeof buf, "plane %dx%d angles %dx%d %s %s", c->Ny + 1, c->Nz + 1, c->Nmu, c->Nom,
                  stream_transport(c) ? "row-streaming" : cluster_transport(c) ? "cluster" : "whole-plane",
                  (c->p.flags & BFPN_FLAG_EQ15_STRAGGLING) ? "eq15+straggling" : "eq15");
    return buf;
}

}  // namespace bfpn
