// Bundles: beams of one shape class advanced together (bfpn_bundle_* in
// include/bfpn_capi.h).  No counterpart in the reference, which runs one beam
// per process (main.cu:344-348).
//
// Each slot of a bundle is a full solver context (its own state, tables, beam,
// IDD history), built by the single-beam entry points.  What the bundle adds
// is the step: instead of each beam launching its own ~20 kernels per depth
// step, the bundle launches each operator ONCE for all slots -- the energy
// sweep, the transport half-steps and the DST of both arrays of every slot
// take a device table of per-slot arguments and each block looks up the slot
// it serves (kernels_step.cu: *_slots_kernel).  Small beams, which leave most
// of a B200 idle on their own (a 17 x 17 x 144-lane plane is 163 energy
// blocks), fill it together; large beams lose nothing.  The secondary source
// (the tensor-core GEMMs) stays per slot, on parallel graph branches.
//
// The step sequence of the current slot set is captured once as a CUDA graph
// and replayed until a slot joins, leaves or takes its first step.  Kernel
// variants -- angles per whole-plane transport block, DST ring depth, energy
// kernel form -- are timed per shape class on the first bundle step of that
// class and the fastest kept for the process (autotuning); every variant
// computes the same values (the energy forms differ only in the order of the
// IDD partial sums).

#include "../../include/bfpn_capi.h"
#include "common.cuh"
#include "context.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

using namespace bfpn;

namespace {

constexpr int kMaxSideStreams = 4;
constexpr int kBundleMaxPlane = 65;  // Ny + 1 and Nz + 1 of a bundle's beams

struct Tuning {
    bool tuned = false;
    int tr_ac = 16;       // angles per whole-plane transport block (8 or 16)
    int dst_stages = 2;   // DST ring stages (2 or 3)
    bool ring = true;     // energy: 4-lane ring kernel (else the 2-lane register kernel)
    std::string report;
};

std::mutex g_tune_mutex;
std::map<std::string, Tuning> g_tune;  // by shape class

thread_local std::string g_bundle_error;

struct Slot {
    bfpn_ctx* ctx = nullptr;
    int nsteps = 0;
    bool running() const { return ctx && ctx->steps_done < nsteps; }
};

// Offsets of one launch's argument and begin tables inside the device image.
struct LaunchTable {
    size_t args = 0, begin = 0;
    int n = 0;            // entries
    long long work = 0;   // blocks (tiles for the DST)
};

struct Plan {
    std::vector<int> prim, sec;  // slots in the primary / secondary halves
    LaunchTable e0a, e0b, e1a, e1b, t0, t1, a0, a1;
    size_t fin = 0;
    int n_fin = 0;
};

}  // namespace

struct bfpn_bundle {
    int device = 0;
    std::vector<Slot> slots;
    cudaStream_t stream = nullptr;
    cudaStream_t side[kMaxSideStreams] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kMaxSideStreams] = {};
    cudaEvent_t ev[8] = {};
    int* err = nullptr;  // device error word of the DST's bounded waits
    // shape class, fixed by the first beam
    bool shaped = false;
    std::string key;
    int NP = 0, N = 0, NA = 0, mode = EMODE_EQ15, cl = 0;
    bool row_stream = false;  // row-streaming transport (else cl > 0: cluster, else whole-plane)
    long long lanes = 0;
    bool no_clip = false;
    Tuning tune;
    bool autotune = true;
    // device argument image and the graph of the current slot set
    void* dimg = nullptr;
    size_t dimg_bytes = 0;
    Plan plan;
    std::string plan_sig;
    cudaGraphExec_t exec = nullptr;
    std::string err_msg;
};

namespace {

bfpn_status bfail(bfpn_bundle* b, bfpn_status s, const std::string& msg) {
    if (b) b->err_msg = msg;
    g_bundle_error = msg;
    return s;
}

#define BUNDLE_CUDA(b, call)                                                                             \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) return bfail(b, BFPN_CUDA_ERROR, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        cudaSetDevice(dev);
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// Blocks of one slot entry in each launch.
int energy_blocks(const bfpn_bundle* b) { return energy_grid(b->lanes, 128); }
long long transport_blocks(const bfpn_bundle* b, int Ng) {
    if (b->row_stream) return static_cast<long long>(Ng) * ((b->NA + 7) / 8);
    if (b->cl) return static_cast<long long>(Ng) * ((b->NA + 7) / 8) * b->cl;
    return static_cast<long long>(Ng) * ((b->NA + b->tune.tr_ac - 1) / b->tune.tr_ac);
}
// Host image of the argument tables, appended with 16-byte alignment.
struct Image {
    std::vector<unsigned char> bytes;
    template <typename A>
    size_t put(const std::vector<A>& v) {
        size_t off = (bytes.size() + 15) / 16 * 16;
        bytes.resize(off + std::max<size_t>(1, v.size()) * sizeof(A));
        if (!v.empty()) std::memcpy(bytes.data() + off, v.data(), v.size() * sizeof(A));
        return off;
    }
};

template <typename A, typename F>
LaunchTable add_table(Image& img, const std::vector<A>& args, F&& work_of) {
    LaunchTable t;
    std::vector<int> begin(args.size() + 1, 0);
    long long total = 0;
    for (size_t i = 0; i < args.size(); ++i) {
        begin[i] = static_cast<int>(total);
        total += work_of(args[i]);
    }
    begin[args.size()] = static_cast<int>(total);
    t.args = img.put(args);
    t.begin = img.put(begin);
    t.n = static_cast<int>(args.size());
    t.work = total;
    return t;
}

// Argument tables for the slots running now; sec = those past their first step.
bfpn_status build_plan(bfpn_bundle* b, const std::vector<int>& prim, const std::vector<int>& sec) {
    Image img;
    Plan p;
    p.prim = prim;
    p.sec = sec;
    const long long eb = energy_blocks(b);
    auto energy = [&](const std::vector<int>& list, int species, bool src, bool partials) {
        std::vector<EnergyArgs<float>> v;
        for (int s : list) {
            bfpn_ctx* c = b->slots[s].ctx;
            v.push_back(bundle_energy_args(c, species, src, partials ? bundle_partials(c, species) : nullptr));
        }
        return add_table(img, v, [&](const EnergyArgs<float>&) { return eb; });
    };
    auto transport = [&](const std::vector<int>& list, int species) {
        std::vector<TransportArgs<float>> v;
        for (int s : list) {
            bfpn_ctx* c = b->slots[s].ctx;
            // psi^1 of the primary keeps its sign only with --no-spatial-clipping; F1 is always clipped
            v.push_back(bundle_transport_args(c, species, 0, species == 0 && b->no_clip));
            v.push_back(bundle_transport_args(c, species, 1, true));
        }
        return add_table(img, v, [&](const TransportArgs<float>& a) { return transport_blocks(b, a.Ng); });
    };
    auto angle = [&](const std::vector<int>& list, int species) {
        std::vector<AngleArgs<float>> v;
        for (int s : list) {
            bfpn_ctx* c = b->slots[s].ctx;
            v.push_back(bundle_angle_args(c, species, 0, b->err));
            v.push_back(bundle_angle_args(c, species, 1, b->err));
        }
        const int SL = angle_slots_tile(b->N);
        return add_table(img, v, [&](const AngleArgs<float>& a) {
            return (static_cast<long long>(a.Ng) * a.nyz + SL - 1) / SL;
        });
    };
    p.e0a = energy(prim, 0, false, false);
    p.t0 = transport(prim, 0);
    p.a0 = angle(prim, 0);
    p.e0b = energy(prim, 0, false, true);
    p.e1a = energy(sec, 1, true, false);
    p.t1 = transport(sec, 1);
    p.a1 = angle(sec, 1);
    p.e1b = energy(sec, 1, true, true);
    std::vector<IddFinalArgs> fin;
    for (int s : prim) {
        const bool has_sec = std::find(sec.begin(), sec.end(), s) != sec.end();
        fin.push_back(bundle_finalize_args(b->slots[s].ctx, has_sec));
    }
    p.fin = img.put(fin);
    p.n_fin = static_cast<int>(fin.size());
    for (const LaunchTable* t : {&p.e0a, &p.t0, &p.a0, &p.e0b, &p.e1a, &p.t1, &p.a1, &p.e1b})
        if (t->work > 0x7fffffffLL) return bfail(b, BFPN_INVALID_ARG, "bundle: too many blocks in one launch");
    // the previous graph may still read the old image
    BUNDLE_CUDA(b, cudaStreamSynchronize(b->stream));
    if (img.bytes.size() > b->dimg_bytes) {
        if (b->dimg) cudaFree(b->dimg);
        b->dimg = nullptr;
        b->dimg_bytes = 0;
        const size_t cap = std::max<size_t>(img.bytes.size() * 2, 4096);
        BUNDLE_CUDA(b, cudaMalloc(&b->dimg, cap));
        b->dimg_bytes = cap;
    }
    // on the bundle's own stream: a plain cudaMemcpy from pageable memory may
    // return before its DMA lands and runs on the legacy stream, which the
    // bundle's non-blocking stream does not wait for -- the next step's
    // kernels could read the previous slot set's arguments
    BUNDLE_CUDA(b, cudaMemcpyAsync(b->dimg, img.bytes.data(), img.bytes.size(), cudaMemcpyHostToDevice, b->stream));
    BUNDLE_CUDA(b, cudaStreamSynchronize(b->stream));
    b->plan = p;
    return BFPN_OK;
}

template <typename A>
const A* at(const bfpn_bundle* b, size_t off) {
    return reinterpret_cast<const A*>(static_cast<const unsigned char*>(b->dimg) + off);
}
const int* begin_of(const bfpn_bundle* b, const LaunchTable& t) { return at<int>(b, t.begin); }

cudaError_t enq_energy_t(bfpn_bundle* b, const LaunchTable& t, cudaStream_t s) {
    return launch_energy_slots(at<EnergyArgs<float>>(b, t.args), begin_of(b, t), t.n, static_cast<int>(t.work),
                               b->mode, b->tune.ring, 128, s);
}
cudaError_t enq_transport_t(bfpn_bundle* b, const LaunchTable& t, cudaStream_t s) {
    if (b->row_stream)
        return launch_transport_stream_slots(at<TransportArgs<float>>(b, t.args), begin_of(b, t), t.n,
                                             static_cast<int>(t.work), b->NP - 1, b->NA, s);
    return launch_transport_slots(at<TransportArgs<float>>(b, t.args), begin_of(b, t), t.n, static_cast<int>(t.work),
                                  b->NP, b->NA, b->tune.tr_ac, b->cl > 0, s);
}
cudaError_t enq_angle_t(bfpn_bundle* b, const LaunchTable& t, cudaStream_t s) {
    return launch_angle_slots(at<AngleArgs<float>>(b, t.args), begin_of(b, t), t.n, t.work, b->N,
                              b->tune.dst_stages, s);
}

// Kernel classes timed by the autotuner.
enum { TK_ENERGY = 0, TK_TRANSPORT = 1, TK_ANGLE = 2, TK_N = 3 };

// One depth step of the planned slots on b->stream.  times != null: eager,
// each timed class bracketed by events and its milliseconds added.
cudaError_t enq_bundle_step(bfpn_bundle* b, double* times) {
    const Plan& p = b->plan;
    cudaStream_t s = b->stream;
    cudaError_t e;
    auto timed = [&](int cls, auto&& launch) -> cudaError_t {
        if (!times) return launch();
        cudaError_t r = cudaEventRecord(b->ev[0], s);
        if (r == cudaSuccess) r = launch();
        if (r == cudaSuccess) r = cudaEventRecord(b->ev[1], s);
        if (r == cudaSuccess) r = cudaEventSynchronize(b->ev[1]);
        float ms = 0.f;
        if (r == cudaSuccess) r = cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]);
        times[cls] += ms;
        return r;
    };
    auto half = [&](const LaunchTable& ea, const LaunchTable& tt, const LaunchTable& aa, const LaunchTable& ebb) {
        cudaError_t r;
        if ((r = timed(TK_ENERGY, [&] { return enq_energy_t(b, ea, s); })) != cudaSuccess) return r;
        if ((r = timed(TK_TRANSPORT, [&] { return enq_transport_t(b, tt, s); })) != cudaSuccess) return r;
        if ((r = timed(TK_ANGLE, [&] { return enq_angle_t(b, aa, s); })) != cudaSuccess) return r;
        if ((r = timed(TK_TRANSPORT, [&] { return enq_transport_t(b, tt, s); })) != cudaSuccess) return r;
        return timed(TK_ENERGY, [&] { return enq_energy_t(b, ebb, s); });
    };
    if ((e = half(p.e0a, p.t0, p.a0, p.e0b)) != cudaSuccess) return e;
    if (!p.sec.empty()) {
        // each slot's source from its primary, on parallel branches
        const int k = std::min<int>(kMaxSideStreams, static_cast<int>(p.sec.size()));
        if ((e = cudaEventRecord(b->ev_fork, s)) != cudaSuccess) return e;
        for (int i = 0; i < k; ++i)
            if ((e = cudaStreamWaitEvent(b->side[i], b->ev_fork, 0)) != cudaSuccess) return e;
        for (size_t j = 0; j < p.sec.size(); ++j)
            if ((e = bundle_source(b->slots[p.sec[j]].ctx, b->side[j % k])) != cudaSuccess) return e;
        for (int i = 0; i < k; ++i) {
            if ((e = cudaEventRecord(b->ev_join[i], b->side[i])) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(s, b->ev_join[i], 0)) != cudaSuccess) return e;
        }
        if ((e = half(p.e1a, p.t1, p.a1, p.e1b)) != cudaSuccess) return e;
    }
    return launch_finalize_idd_slots(at<IddFinalArgs>(b, p.fin), p.n_fin, s);
}

std::string plan_signature(const std::vector<int>& prim, const std::vector<int>& sec, const Tuning& t) {
    std::string sig;
    for (int s : prim) sig += std::to_string(s) + ",";
    sig += "|";
    for (int s : sec) sig += std::to_string(s) + ",";
    sig += "|" + std::to_string(t.tr_ac) + "," + std::to_string(t.dst_stages) + "," + (t.ring ? "r" : "g");
    return sig;
}

void drop_graph(bfpn_bundle* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    b->plan_sig.clear();
}

bfpn_status ensure_plan(bfpn_bundle* b, const std::vector<int>& prim, const std::vector<int>& sec, bool graph) {
    const std::string sig = plan_signature(prim, sec, b->tune);
    if (sig == b->plan_sig && (!graph || b->exec)) return BFPN_OK;
    drop_graph(b);
    bfpn_status st = build_plan(b, prim, sec);
    if (st != BFPN_OK) return st;
    if (graph) {
        BUNDLE_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = enq_bundle_step(b, nullptr);
        cudaGraph_t g = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return bfail(b, BFPN_CUDA_ERROR, std::string("bundle step capture: ") +
                                                 cudaGetErrorString(e != cudaSuccess ? e : e2));
        }
        e = cudaGraphInstantiate(&b->exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return bfail(b, BFPN_CUDA_ERROR, std::string("bundle graph: ") + cudaGetErrorString(e));
    }
    b->plan_sig = sig;
    return BFPN_OK;
}

// Autotuning: two eager steps per variant set, A and B alternating (A B A B),
// each kernel class keeps its faster variant.  The steps are real steps of
// the bundle.  Returns the steps taken.
bfpn_status autotune(bfpn_bundle* b, const std::vector<int>& prim, int max_steps, int* taken) {
    *taken = 0;
    Tuning A = b->tune, B = b->tune;
    A.tr_ac = 16;
    B.tr_ac = 8;
    A.dst_stages = 2;
    B.dst_stages = 3;
    A.ring = true;
    B.ring = false;
    double tA[TK_N] = {}, tB[TK_N] = {};
    const int rounds = std::min(4, max_steps);
    for (int r = 0; r < rounds; ++r) {
        b->tune = (r % 2 == 0) ? A : B;
        // a slot's first step has no secondary half
        std::vector<int> sec_now;
        for (int s : prim)
            if (b->slots[s].ctx->steps_done > 0) sec_now.push_back(s);
        bfpn_status st = ensure_plan(b, prim, sec_now, false);
        if (st != BFPN_OK) return st;
        cudaError_t e = enq_bundle_step(b, (r % 2 == 0) ? tA : tB);
        if (e != cudaSuccess) return bfail(b, BFPN_CUDA_ERROR, std::string("bundle tuning step: ") + cudaGetErrorString(e));
        for (int s : prim) b->slots[s].ctx->steps_done += 1;
        ++*taken;
        b->plan_sig.clear();
    }
    Tuning best = A;
    if (rounds >= 2) {
        const bool fixed_tr = b->cl || b->row_stream;  // one transport form: nothing to choose
        best.tr_ac = (fixed_tr || tA[TK_TRANSPORT] <= tB[TK_TRANSPORT]) ? A.tr_ac : B.tr_ac;
        best.dst_stages = tA[TK_ANGLE] <= tB[TK_ANGLE] ? A.dst_stages : B.dst_stages;
        best.ring = tA[TK_ENERGY] <= tB[TK_ENERGY] ? A.ring : B.ring;
        best.tuned = true;
        char buf[320];
        std::snprintf(buf, sizeof buf,
                      "%s: transport %s (%.3f ms vs %.3f ms per step-pair), DST %d stages (%.3f vs %.3f), "
                      "energy %s (%.3f vs %.3f)",
                      b->key.c_str(),
                      b->row_stream ? "row-streaming" : b->cl ? "cluster" : (best.tr_ac == 16 ? "16 angles/block" : "8 angles/block"),
                      tA[TK_TRANSPORT], tB[TK_TRANSPORT], best.dst_stages, tA[TK_ANGLE], tB[TK_ANGLE],
                      best.ring ? "4-lane ring" : "2-lane register", tA[TK_ENERGY], tB[TK_ENERGY]);
        best.report = buf;
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tune[b->key] = best;
    }
    b->tune = best;
    return BFPN_OK;
}

}  // namespace

extern "C" {

bfpn_status bfpn_bundle_accepts(const bfpn_beam* beam) {
    if (!beam) return bfail(nullptr, BFPN_INVALID_ARG, "bundle: null beam");
    const bfpn_grid& g = beam->grid;
    const uint32_t fl = beam->phys.flags;
    if (beam->precision != BFPN_PREC_MIXED) return bfail(nullptr, BFPN_INVALID_ARG, "bundle: mixed-precision beams only");
    if (fl & (BFPN_FLAG_ENERGY_ONLY | BFPN_FLAG_PRIMARY_ONLY | BFPN_FLAG_NO_TRANSPORT | BFPN_FLAG_NO_ANGLE |
              BFPN_FLAG_LEGACY_ENERGY | BFPN_FLAG_LITE_MEMORY | BFPN_FLAG_STREAMING_FULL))
        return bfail(nullptr, BFPN_INVALID_ARG, "bundle: the eq15 step with transport, angular diffusion and secondaries only");
    // paired angles share direction signs when each half of a row of angles has an even count
    const int N = g.Nom;
    if (g.Nmu != N || N % 4 != 0 || N > 32)
        return bfail(nullptr, BFPN_INVALID_ARG, "bundle: square angular grids with Nom = Nmu a multiple of 4 up to 32");
    const long long nyz = static_cast<long long>(g.Ny + 1) * (g.Nz + 1);
    if (g.Ny < 1 || g.Nz < 1 || nyz < angle_slots_tile(N))
        return bfail(nullptr, BFPN_INVALID_ARG, "bundle: the plane is smaller than one DST tile");
    // planes up to 65 x 65 points: a larger beam (the 80 x 80 paper grid holds
    // 1.3e9 cells per array) fills the GPU alone, so it gains nothing from a
    // bundle and runs on its own context
    if (g.Ny + 1 > kBundleMaxPlane || g.Nz + 1 > kBundleMaxPlane)
        return bfail(nullptr, BFPN_INVALID_ARG, "bundle: planes up to 65 x 65 points; larger beams run alone");
    const bool square_plane = g.Ny == g.Nz && (transport_plane_supported(g.Ny, g.Nz) || transport_cluster_supported(g.Ny, g.Nz));
    if (!transport_stream_supported(g.Ny, N * N) && !square_plane)
        return bfail(nullptr, BFPN_INVALID_ARG, "bundle: no batched transport kernel for this plane");
    return BFPN_OK;
}

const char* bfpn_bundle_last_error(const bfpn_bundle* b) { return b ? b->err_msg.c_str() : g_bundle_error.c_str(); }

bfpn_status bfpn_bundle_create(int32_t device, int32_t max_slots, bfpn_bundle** out) {
    if (!out || max_slots <= 0 || max_slots > 4096) return bfail(nullptr, BFPN_INVALID_ARG, "bundle: bad arguments");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return bfail(nullptr, BFPN_NO_DEVICE, "bundle: no such device");
    }
    DeviceScope scope(device);
    auto* b = new bfpn_bundle();
    b->device = device;
    b->slots.resize(max_slots);
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    for (int i = 0; e == cudaSuccess && i < kMaxSideStreams; ++i) {
        e = cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
    for (int i = 0; e == cudaSuccess && i < 8; ++i) e = cudaEventCreate(&b->ev[i]);
    if (e == cudaSuccess) e = cudaMalloc(&b->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(b->err, 0, sizeof(int), b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) {
        const std::string msg = std::string("bundle: ") + cudaGetErrorString(e);
        bfpn_bundle_destroy(b);
        return bfail(nullptr, BFPN_CUDA_ERROR, msg);
    }
    *out = b;
    return BFPN_OK;
}

bfpn_status bfpn_bundle_set_option(bfpn_bundle* b, int32_t option, int32_t value) {
    if (!b) return bfail(nullptr, BFPN_INVALID_ARG, "bundle: null");
    if (option == BFPN_BUNDLE_OPT_AUTOTUNE) {
        b->autotune = value != 0;
        return BFPN_OK;
    }
    Tuning t = b->tune;
    if (option == BFPN_BUNDLE_OPT_TRANSPORT_ANGLES && (value == 8 || value == 16)) t.tr_ac = value;
    else if (option == BFPN_BUNDLE_OPT_DST_STAGES && (value == 2 || value == 3)) t.dst_stages = value;
    else if (option == BFPN_BUNDLE_OPT_ENERGY_RING) t.ring = value != 0;
    else return bfail(b, BFPN_INVALID_ARG, "bundle: unknown option or value");
    t.tuned = true;
    t.report = b->key + ": set by the caller";
    b->tune = t;
    b->autotune = false;
    drop_graph(b);
    return BFPN_OK;
}

bfpn_status bfpn_bundle_admit(bfpn_bundle* b, const bfpn_beam* beam, int32_t* slot_out) {
    if (!b || !beam || !slot_out) return bfail(b, BFPN_INVALID_ARG, "bundle admit: null argument");
    *slot_out = -1;
    if (beam->precision != BFPN_PREC_MIXED) return bfail(b, BFPN_INVALID_ARG, "bundle admit: a bundle holds mixed-precision beams");
    if (beam->nsteps < 1) return bfail(b, BFPN_INVALID_ARG, "bundle admit: nsteps must be >= 1");
    int free_slot = -1;
    for (size_t i = 0; i < b->slots.size(); ++i)
        if (!b->slots[i].ctx) {
            free_slot = static_cast<int>(i);
            break;
        }
    if (free_slot < 0) return bfail(b, BFPN_INVALID_ARG, "bundle admit: every slot is taken");
    if (b->shaped && (beam->grid.Ny + 1 != b->NP || beam->grid.Nz + 1 != b->NP || beam->grid.Nmu != b->N ||
                      beam->grid.Nom != b->N))
        return bfail(b, BFPN_INVALID_ARG, "bundle admit: the beam's grid is not the bundle's shape class (" + b->key + ")");
    if (bfpn_bundle_accepts(beam) != BFPN_OK)
        return bfail(b, BFPN_INVALID_ARG, std::string("bundle admit: ") + g_bundle_error.substr(8));
    DeviceScope scope(b->device);
    // admission by footprint: the whole context must fit in free memory, with a margin
    uint64_t need = 0;
    bfpn_status st = bfpn_footprint_bytes(&beam->grid, &beam->phys, BFPN_PREC_MIXED, &need);
    if (st != BFPN_OK) return bfail(b, st, std::string("bundle admit: ") + bfpn_last_error(nullptr));
    size_t free_b = 0, total_b = 0;
    BUNDLE_CUDA(b, cudaMemGetInfo(&free_b, &total_b));
    const uint64_t margin = 512ull << 20;
    if (need + margin > free_b) {
        char msg[160];
        std::snprintf(msg, sizeof msg, "bundle admit: the beam needs %.2f GiB, %.2f GiB free", need / 1073741824.0,
                      free_b / 1073741824.0);
        return bfail(b, BFPN_OOM, msg);
    }
    bfpn_ctx* c = nullptr;
    if ((st = bfpn_create(&beam->grid, &beam->phys, BFPN_PREC_MIXED, b->device, &c)) != BFPN_OK)
        return bfail(b, st, std::string("bundle admit: ") + bfpn_last_error(nullptr));
    auto undo = [&](bfpn_status s2, const std::string& m) {
        const std::string msg = "bundle admit: " + m;
        bfpn_destroy(c);
        return bfail(b, s2, msg);
    };
    if ((st = bfpn_load_tables(c, beam->mu, beam->mu_rows, beam->sigma_c, beam->sigma_rows)) != BFPN_OK)
        return undo(st, bfpn_last_error(c));
    if ((st = bfpn_init_beam(c)) != BFPN_OK) return undo(st, bfpn_last_error(c));
    const std::string why = bundle_ready(c);
    if (!why.empty()) return undo(BFPN_INVALID_ARG, why);
    // a beam whose tensor-core source buffers did not fit waits for memory like one that does not fit at all
    if (!bundle_tc_source(c)) return undo(BFPN_OOM, "no room for the tensor-core source buffers");
    const std::string key = bundle_class_key(c);
    const int mode = (c->p.flags & BFPN_FLAG_EQ15_STRAGGLING) ? EMODE_EQ15_STRAG : EMODE_EQ15;
    const bool no_clip = (c->p.flags & BFPN_FLAG_NO_SPATIAL_CLIPPING) != 0;
    if (b->shaped && (key != b->key || mode != b->mode || no_clip != b->no_clip))
        return undo(BFPN_INVALID_ARG, "the beam's kernels (" + key + ") are not the bundle's (" + b->key + ")");
    if ((st = bundle_reserve_history(c, beam->nsteps)) != BFPN_OK) return undo(st, bfpn_last_error(c));
    if (!b->shaped) {
        b->shaped = true;
        b->key = key;
        b->NP = c->Ny + 1;
        b->N = c->Nom;
        b->NA = c->NA;
        b->lanes = c->per_e;
        b->mode = mode;
        b->no_clip = no_clip;
        b->cl = bundle_cluster_size(c);
        b->row_stream = bundle_stream_transport(c);
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) b->tune = it->second;
    }
    b->slots[free_slot].ctx = c;
    b->slots[free_slot].nsteps = beam->nsteps;
    *slot_out = free_slot;
    return BFPN_OK;
}

bfpn_status bfpn_bundle_step(bfpn_bundle* b, int32_t nsteps) {
    if (!b || nsteps < 0) return bfail(b, BFPN_INVALID_ARG, "bundle step: bad arguments");
    DeviceScope scope(b->device);
    int left = nsteps;
    while (left > 0) {
        std::vector<int> prim, sec;
        int min_rest = left;
        for (size_t i = 0; i < b->slots.size(); ++i) {
            const Slot& s = b->slots[i];
            if (!s.running()) continue;
            prim.push_back(static_cast<int>(i));
            if (s.ctx->steps_done > 0) sec.push_back(static_cast<int>(i));
            min_rest = std::min(min_rest, s.nsteps - s.ctx->steps_done);
        }
        if (prim.empty()) break;
        if (b->autotune && !b->tune.tuned) {
            int taken = 0;
            bfpn_status st = autotune(b, prim, min_rest, &taken);
            if (st != BFPN_OK) return st;
            left -= taken;
            continue;
        }
        // a slot's first step has no secondary half: one step with that plan
        const int k = (sec.size() < prim.size()) ? 1 : min_rest;
        bfpn_status st = ensure_plan(b, prim, sec, true);
        if (st != BFPN_OK) return st;
        for (int i = 0; i < k; ++i) BUNDLE_CUDA(b, cudaGraphLaunch(b->exec, b->stream));
        for (int s : prim) b->slots[s].ctx->steps_done += k;
        left -= k;
    }
    return BFPN_OK;
}

bfpn_status bfpn_bundle_sync(bfpn_bundle* b) {
    if (!b) return bfail(nullptr, BFPN_INVALID_ARG, "bundle: null");
    DeviceScope scope(b->device);
    BUNDLE_CUDA(b, cudaStreamSynchronize(b->stream));
    int err = 0;
    BUNDLE_CUDA(b, cudaMemcpy(&err, b->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
        cudaMemsetAsync(b->err, 0, sizeof(int), b->stream);
        cudaStreamSynchronize(b->stream);
        return bfail(b, BFPN_TIMEOUT, "bundle: a kernel's bounded wait ran out (code " + std::to_string(err) + ")");
    }
    // the slots' own error words (the tensor-core source kernels' bounded waits)
    for (size_t i = 0; i < b->slots.size(); ++i) {
        bfpn_ctx* c = b->slots[i].ctx;
        if (!c || !c->dev_err) continue;
        BUNDLE_CUDA(b, cudaMemcpy(&err, c->dev_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) {
            cudaMemsetAsync(c->dev_err, 0, sizeof(int), b->stream);
            cudaStreamSynchronize(b->stream);
            return bfail(b, BFPN_TIMEOUT, "bundle: slot " + std::to_string(i) + ": a source kernel's bounded wait ran out "
                                          "(code " + std::to_string(err) + ")");
        }
    }
    return BFPN_OK;
}

int32_t bfpn_bundle_running(const bfpn_bundle* b) {
    if (!b) return -1;
    int n = 0;
    for (const Slot& s : b->slots) n += s.running() ? 1 : 0;
    return n;
}

bfpn_status bfpn_bundle_slot(const bfpn_bundle* b, int32_t slot, int32_t* steps_done, int32_t* nsteps) {
    if (!b || slot < 0 || slot >= static_cast<int>(b->slots.size()))
        return bfail(nullptr, BFPN_INVALID_ARG, "bundle slot: out of range");
    const Slot& s = b->slots[slot];
    if (steps_done) *steps_done = s.ctx ? s.ctx->steps_done : -1;
    if (nsteps) *nsteps = s.ctx ? s.nsteps : 0;
    return BFPN_OK;
}

bfpn_status bfpn_bundle_collect(bfpn_bundle* b, int32_t slot, double* idd, double* proxy, int32_t capacity) {
    if (!b || slot < 0 || slot >= static_cast<int>(b->slots.size()) || !b->slots[slot].ctx)
        return bfail(b, BFPN_INVALID_ARG, "bundle collect: empty or bad slot");
    Slot& s = b->slots[slot];
    if (s.running()) return bfail(b, BFPN_INVALID_ARG, "bundle collect: the slot has steps left");
    if ((idd || proxy) && capacity < s.nsteps) return bfail(b, BFPN_INVALID_ARG, "bundle collect: capacity < nsteps");
    bfpn_status st = bfpn_bundle_sync(b);
    if (st != BFPN_OK) return st;
    if (idd || proxy) {
        if ((st = bfpn_history_download(s.ctx, 0, s.nsteps, idd, proxy)) != BFPN_OK)
            return bfail(b, st, std::string("bundle collect: ") + bfpn_last_error(s.ctx));
    }
    drop_graph(b);
    bfpn_destroy(s.ctx);
    s = Slot{};
    return BFPN_OK;
}

int32_t bfpn_bundle_tuning(const bfpn_bundle* b, char* buf, int32_t buf_len) {
    if (!b || !buf || buf_len <= 0) return -1;
    const std::string& r = b->tune.report.empty() ? std::string("not tuned") : b->tune.report;
    const int n = std::snprintf(buf, buf_len, "%s", r.c_str());
    return n < buf_len ? n : buf_len - 1;
}

void* bfpn_bundle_stream(bfpn_bundle* b) { return b ? static_cast<void*>(b->stream) : nullptr; }

bfpn_status bfpn_bundle_destroy(bfpn_bundle* b) {
    if (!b) return BFPN_OK;
    DeviceScope scope(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (Slot& s : b->slots)
        if (s.ctx) bfpn_destroy(s.ctx);
    drop_graph(b);
    if (b->dimg) cudaFree(b->dimg);
    if (b->err) cudaFree(b->err);
    for (int i = 0; i < kMaxSideStreams; ++i) {
        if (b->side[i]) cudaStreamDestroy(b->side[i]);
        if (b->ev_join[i]) cudaEventDestroy(b->ev_join[i]);
    }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    for (cudaEvent_t& e : b->ev)
        if (e) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return BFPN_OK;
}

}  // extern "C"
