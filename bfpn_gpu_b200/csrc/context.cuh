// Internal: the solver context behind the C ABI's bfpn_ctx handle, shared by
// capi.cu (single beams) and bundle.cu (beams of one shape class advanced
// together).  Not part of the public interface.
#pragma once

#include "../../include/bfpn_capi.h"
#include "common.cuh"
#include "tables.hpp"

#include <string>
#include <vector>

namespace bfpn {

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace bfpn

struct bfpn_ctx {
    bfpn_grid g{};
    bfpn_phys p{};
    int prec = BFPN_PREC_FP64;
    int device = 0;
    size_t elem = 8;
    bfpn::Deltas d{};
    int Ng = 0, Ny = 0, Nz = 0, Nmu = 0, Nom = 0, nyz = 0, NA = 0;
    long long per_e = 0, cells = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    std::vector<bfpn::DevBuf> allocs;
    void* st[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    void* tmp = nullptr;       // out-of-place transport target (tiled planes only)
    void* src = nullptr;       // secondary source
    void* A1 = nullptr;        // angular contractions of the primary (one block of a_bytes; A2 inside it,
    void* A2 = nullptr;        // or the whole block in the tensor-core operand layout)
    size_t a_bytes = 0;
    double* ecoef_half = nullptr;   // energy constants for dt/2
    double* ecoef_op = nullptr;     // energy constants for a per-operator dt
    double ecoef_op_dt = -1.0;
    double* dose_coef = nullptr;
    void* omega = nullptr;
    void* fac_step = nullptr;       // angle factor for the full step dt
    void* fac_op = nullptr;         // angle factor for a per-operator dt
    double fac_op_dt = -1.0;
    void* sine_u = nullptr;
    void* sine_v = nullptr;
    void* ker_v = nullptr;
    double* e1 = nullptr;
    double* e2 = nullptr;
    int* groups = nullptr;
    int n_groups = 0;
    int* tile_lo = nullptr;
    int* tile_hi = nullptr;
    int tile_e = 16;
    double* beam_yza = nullptr;
    double* beam_e = nullptr;
    double* partials = nullptr;     // [2][energy_grid][2]
    int n_part = 0;
    double* hist_idd = nullptr;
    double* hist_proxy = nullptr;
    int hist_cap = 0;
    int* counter = nullptr;
    int* zero_counter = nullptr;    // scratch counter for one-off IDD reductions
    int* dev_err = nullptr;         // device error word (bounded waits that ran out)
    void* bblob = nullptr;          // split-bf16 angular kernel tiles for the tensor-core source
    void* ablob = nullptr;          // packed split-bf16 A operand (pipelined tensor-core source)
    void* eblob = nullptr;          // split-bf16 energy coefficient tiles (tensor-core source)
    int4* ulist = nullptr;          // non-zero k chunks / column ranges of the angular kernel blocks
    int* ubegin = nullptr;          // [n_groups * umma_ntiles + 1] offsets into ulist
    int* ework = nullptr;           // energy work items {chunk, column, columns, e group}
    int* ework_begin = nullptr;     // [e tiles + 1]
    int e_et = 0, e_emax = 0;
    bool use_umma = true;
    int umma_nt = 0, umma_bk = 16, umma_ntiles = 0;
    double* scalar_out = nullptr;   // [2] one-off IDD / proxy
    double* moments = nullptr;      // [Ng][2]
    double* plane = nullptr;        // [nyz] spot dose plane
    bool lite = false;              // lite-memory mode: psi^1 of the primary only
    // out-of-core mode: st[][] are pinned host arrays; device chunk buffers
    bool ooc = false;
    int ooc_lane_req = 262144, ooc_group_req = 128;  // requested chunk sizes (lanes, groups)
    int lc_pos = 0, lc = 0, n_lc = 0, ecg = 0;        // positions / lanes per lane chunk, lane chunks, groups per group chunk
    bool ooc_ready = false;
    void* dl[2][4] = {};    // two slots of a lane chunk: the species' psi^1, psi^2; the primary's for the source
    void* dgc[2] = {};      // two slots of a group chunk
    cudaStream_t s_in = nullptr, s_out = nullptr;        // host-to-device / device-to-host copies
    cudaEvent_t ev_in[2] = {}, ev_comp[2] = {}, ev_out[2] = {}, ev_pass = nullptr;
    void* ooc_part = nullptr;                            // IDD partials of every lane chunk, both species
    std::vector<void*> host_allocs;
    double* lite_coef = nullptr;    // [Ng][2] lite step constants

    bfpn::BeamTables tables;
    std::vector<double> raw_sigma;  // sigma_c as given, before the optional calibration
    bool tables_loaded = false;
    bool beam_ready = false;
    int steps_done = 0;
    bool secondary_zero = true;

    // transport launch shape
    int tr_ac = 16, tr_ty = 1, tr_tz = 1;
    bool tr_inplace = true;
    bool tr_plane_ok = false;   // a compiled whole-plane kernel exists for this plane
    bool tr_plane = false;      // use it
    int tr_plane_ac = 8;
    bool tr_pairs_ok = false;   // angle pairs share direction signs (float whole planes)
    bool tr_pairs = true;       // use the paired kernel where it applies
    bool tr_cluster_ok = false; // a cluster kernel is compiled for this plane (float state)
    int tr_cluster = 1;         // 0 off, 1 planes without a whole-plane kernel, 2 every supported plane
    bool tr_stream_ok = false;  // the row-streaming kernel applies (float state, plane <= 128 wide)
    int tr_stream = 1;          // 0 off, 1 planes without a whole-plane kernel, 2 every supported plane
    bool tr_tile_ok = false;    // the plane needs tiles: the unrolled tiled kernel applies
    bool tr_tile = false;       // use it
    int tr_tile_ac = 8;
    int ang_slices = 4;
    int energy_block = 128;

    cudaGraphExec_t graph_exec = nullptr;
    int graph_key = -1;
    bool use_graphs = true;
    // overlapped steps: the secondary half of step n (source, energy and
    // transport of the secondary species, the step's IDD) runs on s_sec beside
    // the primary half of step n+1; graph ovl_exec[p] serves steps of parity p
    bool overlap = true;
    bool pending_sec = false;  // the secondary half of step steps_done-1 is still owed
    cudaStream_t s_sec = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_pread = nullptr, ev_join = nullptr;
    // inside an overlapped body the T-A-T chains of psi^2 also get their own
    // streams (one per species): s_f[k], forked / joined by ev_ff[k] / ev_fj[k]
    bool split_tat = false;
    bool split_chains = true;  // option: split the chains in overlapped bodies
    cudaStream_t s_f[2] = {nullptr, nullptr};
    cudaEvent_t ev_ff[2] = {nullptr, nullptr}, ev_fj[2] = {nullptr, nullptr};
    cudaGraphExec_t ovl_exec[2] = {nullptr, nullptr};
    // fused primary energy passes (mixed precision, overlapped steps): the
    // closing pass of step n and the opening pass of step n+1 run as one
    // kernel, which also writes the source's operand.  pending_close: the
    // closing pass and the secondary half of step steps_done-1 are still owed
    // (pending_first: that step is step 0, which has no secondary half)
    bool fuse_energy = true;    // option
    bool pending_close = false, pending_first = false;
    bool src_prepacked = false;  // the source's operand is already in ablob
    int* gmap = nullptr;         // [Ng]: index among the source groups, -1 for none
    cudaGraphExec_t fus_exec[2] = {nullptr, nullptr};
    bool profiling = false;
    struct Pending {
        int cls;
        cudaEvent_t a, b;
    };
    std::vector<cudaEvent_t> ev_pool;
    std::vector<Pending> pending;
    double prof_ms[BFPN_KERNEL_CLASSES] = {};
    int prof_n[BFPN_KERNEL_CLASSES] = {};
    long long launches = 0;        // launches issued by host enqueue code
    int kernels_per_step = 0;

    std::string err;
};


namespace bfpn {

// Per-slot pieces of a depth step, for bundle.cu (capi.cu).  Float state.
// A context qualifies for a bundle when bundle_ready is empty.
std::string bundle_ready(const bfpn_ctx* c);
// The slot's secondary source runs on the tensor-core kernels (its operand
// buffers were allocated); a context that fell back to the CUDA-core source
// for lack of memory does not enter a bundle.
bool bundle_tc_source(const bfpn_ctx* c);
EnergyArgs<float> bundle_energy_args(bfpn_ctx* c, int species, bool with_source, double* partials);
TransportArgs<float> bundle_transport_args(bfpn_ctx* c, int species, int coef, bool preserve_sign);
AngleArgs<float> bundle_angle_args(bfpn_ctx* c, int species, int coef, int* err);
// The secondary source of the context's current primary, enqueued on s.
cudaError_t bundle_source(bfpn_ctx* c, cudaStream_t s);
// IDD partial buffers of a step: the primary's and the secondary's, and
// their counts; the finalisation arguments (secondary = false: the
// secondary contributes nothing, as on the first step).
IddFinalArgs bundle_finalize_args(bfpn_ctx* c, bool secondary);
double* bundle_partials(bfpn_ctx* c, int species);
// Room for n more IDD history entries; drops the context's own step graphs.
bfpn_status bundle_reserve_history(bfpn_ctx* c, int n);
// The shape class of the context's kernels (transport plane / cluster, DST
// size, energy kernel) as a printable key.
std::string bundle_class_key(const bfpn_ctx* c);
// CTAs per cluster of the context's cluster transport, 0 for whole-plane transport.
int bundle_cluster_size(const bfpn_ctx* c);
// The context's transport runs the row-streaming kernel.
bool bundle_stream_transport(const bfpn_ctx* c);

}  // namespace bfpn
