// Shared definitions of the B200 BFPn depth-step kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

namespace bfpn {

// include/config.hpp:38-41 of the reference.
constexpr double kEpsilon = 1e-10;

// Number of double coefficients per energy group in the energy-sweep table
// (see tables.cpp: build_energy_coefficients).
constexpr int kEnergyCoef = 20;
enum EnergyCoef {
    EC_INV_F = 0,      // 1 / max(1/dt + a_lo/2 + sig/2, eps)
    EC_A = 1,          // 1.5 a_hi * inv_F
    EC_F_FROM_F = 2,   // 0.5 a_lo * inv_F
    EC_F_FROM_HI = 3,  // 0.5 a_hi * inv_F
    EC_C_UP = 4,       // 0.5 a_hi          (common term: up)
    EC_C_CUR = 5,      // -0.5 a_lo         (common term: cur)
    EC_C_F = 6,        // 1/dt - 0.5 sig    (common term: F_g)
    EC_R_F = 7,        // coefficient of f_g in rhs1e + rhs2e
    EC_R_UP = 8,       // 1.5 a_hi
    EC_R_CUR = 9,      // 1.5 a_lo
    EC_R_FG = 10,      // -1.5 (a_lo + a_hi)
    EC_R_HI = 11,      // 1.5 a_hi - 0.5 A a_hi
    EC_INV_COE = 12,   // 1 / max(coe, eps)
    EC_S_HI = 13,      // straggling: 0.5 rho T_hi / dg2
    EC_S_LO = 14,      // straggling: 0.5 rho T_lo / dg2
    EC_S_G = 15,       // straggling: rho T_g / dg2
    EC_L_IDT = 16,     // legacy: 1/dt
    EC_L_HI = 17,      // legacy: rho S_hi / dg
    EC_L_INV_DEN = 18, // legacy: 1 / max(denominator, eps)
    EC_L_LAP = 19      // legacy straggling: 0.5 dt T_g / dg2 (0 when off)
};

enum EnergyMode { EMODE_EQ15 = 0, EMODE_EQ15_STRAG = 1, EMODE_LEGACY = 2 };

// 16-byte vector of T for staging loads and stores.
template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; static constexpr int W = 4; };
template <> struct Vec16<double> { using type = double2; static constexpr int W = 2; };

// Arguments of one energy half-step over one species.
template <typename T>
struct EnergyArgs {
    T* F;                  // psi^1, in place
    T* f;                  // psi^2, in place
    const T* src;          // catastrophic source of psi^1, or nullptr
    const double* coef;    // [Ng][kEnergyCoef]
    int Ng;
    long long lanes;       // nyz * NA
    int mode;              // EnergyMode
    // fused IDD (nullptr partials = off)
    double* partials;      // [gridDim.x][2]: dose part, psi^2 part
    const double* dose_coef;  // [Ng][2]: weight of psi^1 and psi^2
    int NA, Ny, Nz;
    int trapezoidal;
    long long lane0 = 0;   // state lane of lane 0 (a chunk of whole positions; trapezoidal weights)
};

// Byte offset of element (row, k) in a K-major no-swizzle UMMA tile of
// `rows` rows: core matrix (row/8, k/8) of 8 x 8 bf16, 16-byte rows.
__host__ __device__ inline size_t umma_kmajor_offset(int row, int k, int rows) {
    return (static_cast<size_t>(k >> 3) * (rows >> 3) + (row >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

// The primary's closing energy half-step of one depth step fused with the
// opening half-step of the next (no source; float state, lanes a multiple of
// 4, eq15 modes).  e.F / e.f hold the state after the step's transport and
// angular diffusion and receive the state after the next step's opening
// half; e.partials receives the closing pass's IDD partials (one pair per
// block, as energy_ring_kernel).  At the midpoint (after the closing pass)
// the state of every source group is also written, split into bf16 hi / lo,
// as the A operand of the source's angular contraction (rows 0..63 of a
// 64-position tile max(psi^1, 0), rows 64..127 psi^2, K-major core layout,
// 16-wide k chunks): the operand pack_source_operand_kernel would build.
struct EnergyFusedArgs {
    EnergyArgs<float> e;
    uint8_t* ablob;      // [n_groups][n_mt][nk][hi|lo][128 x 16 bf16], or nullptr
    const int* gmap;     // [Ng]: index of each group among the source groups, -1 for none
    int n_mt, nk;
};
cudaError_t launch_energy_fused(const EnergyFusedArgs& a, cudaStream_t s);
bool energy_fused_supported(long long lanes, int mode, int NA);

// Arguments of one transport half-step (Eq. 18) over one array.
template <typename T>
struct TransportArgs {
    const T* in;
    T* out;                // == in only when one tile covers a whole plane
    const T* omega;        // [NA][2]: omega_y, omega_z
    int Ny, Nz, NA, Ng;
    T dt, dy, dz;
    int tile_y, tile_z;    // output tile (positions)
    int preserve_sign;
    int pairs = 0;         // float whole planes: two angles per thread (transport_pairs_ok)
};

// Arguments of one angular-diffusion step (Eq. 19) over one array.
template <typename T>
struct AngleArgs {
    T* F;                  // in place
    const T* fac;          // [Ng][NA] CN ratio * 4/((Nom+1)(Nmu+1))
    const T* sine_u;       // [Nom][Nom]
    const T* sine_v;       // [Nmu][Nmu]
    int Nom, Nmu, nyz, Ng;
    int slices_per_block;
    int* err = nullptr;    // device error word: enables the pipelined kernel (bounded waits report here)
    int pairs = 0;         // float state: two lines per thread in the pipelined kernel
};

// Arguments of the factorised catastrophic source.
template <typename T>
struct SourceArgs {
    const T* P1;           // primary psi^1
    const T* P2;           // primary psi^2
    const T* ker_v;        // [Ng][NA][NA]  (src, in, out)
    const int* groups;     // source groups with a non-zero angular kernel that some output uses
    int n_groups;
    T* A1;                 // [Ng][nyz][NA] angular contraction of max(P1, 0)
    T* A2;                 // [Ng][nyz][NA] angular contraction of P2
    T* S;                  // [Ng][nyz][NA] output source
    const double* e1;      // [Ng][Ng] ker_e1, row = output group
    const double* e2;      // [Ng][Ng] ker_e2
    const int* tile_lo;    // per output-group tile: first source group of the union band
    const int* tile_hi;    // per output-group tile: one past the last
    int Ng, nyz, NA;
    double dg;
};

// ---- multi-slot launches (a bundle of beams of one shape class) ----------
// One launch serves several slots: blocks (or work tiles) [begin[s],
// begin[s+1]) belong to slot s and read that slot's argument struct from a
// device array.  begin has nslots + 1 entries, begin[0] = 0.
#ifdef __CUDACC__
__device__ __forceinline__ int find_slot(const int* __restrict__ begin, int nslots, long long b) {
    int lo = 0, hi = nslots - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(begin + mid) <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
#endif

// Arguments of one slot's IDD finalisation (launch_finalize_idd's arguments).
struct IddFinalArgs {
    const double* p;
    int n;
    const double* p2;
    int n2;
    double idd_scale, proxy_scale;
    double* hist_idd;
    double* hist_proxy;
    int* counter;
    int capacity;
};

// Float state only.  args / begin are device arrays; blocks = begin[nslots].
// Dynamic shared memory: raise `func`'s limit, once per device, to the most
// the device allows a block (never lowered afterwards), and check that `need`
// fits.  The limit is a process-wide property of the function; setting it per
// launch to that launch's size let a thread lower it between another
// thread's capture of a larger launch and that graph's replay.
cudaError_t allow_dynamic_smem(const void* func, size_t need);

// Energy sweep: ring = the 4-lane ring kernel (lanes % 4 == 0, not legacy),
// else the register kernel with `block` threads; every slot's grid is that
// kernel's energy_grid of its lanes.
cudaError_t launch_energy_slots(const EnergyArgs<float>* args, const int* begin, int nslots, int blocks, int mode,
                                bool ring, int block, cudaStream_t s);
// Transport of square planes of NP = Ny + 1 points, paired angles: the
// whole-plane kernel with ang_chunk angles per block (NP a compiled plane
// size; slot grid Ng * ceil(NA / ang_chunk)) or, for a compiled cluster size,
// the cluster kernel (slot grid Ng * ceil(NA / 8) * cluster size).
cudaError_t launch_transport_slots(const TransportArgs<float>* args, const int* begin, int nslots, int blocks,
                                   int NP, int NA, int ang_chunk, bool cluster, cudaStream_t s);
int transport_cluster_size(int NP);
// Row-streaming transport (float state, paired angles, Ny + 1 <= 256, any Nz):
// one block per (group, 8-angle chunk) plane walking the z rows, in place.
cudaError_t launch_transport_stream(const TransportArgs<float>& a, cudaStream_t s);
bool transport_stream_supported(int Ny, int NA);
// The same over the slots of a bundle (slot grid Ng * ceil(NA / 8)).
cudaError_t launch_transport_stream_slots(const TransportArgs<float>* args, const int* begin, int nslots, int blocks,
                                          int Ny, int NA, cudaStream_t s);
// Pipelined paired DST (Nom = Nmu = N even): work tiles of 2 * 128 / N slices;
// tile_begin = tile offsets (slot s has ceil(Ng nyz / tile) tiles); stages 2 or 3.
cudaError_t launch_angle_slots(const AngleArgs<float>* args, const int* tile_begin, int nslots, long long tiles,
                               int N, int stages, cudaStream_t s);
int angle_slots_tile(int N);
// IDD finalisation, one block per slot (advance the counters).
cudaError_t launch_finalize_idd_slots(const IddFinalArgs* args, int nslots, cudaStream_t s);

// Launchers (kernels_*.cu).  All return the launch status.
template <typename T> cudaError_t launch_energy(const EnergyArgs<T>& a, int block, cudaStream_t s);
// Lite-memory primary step over psi^1 with fused IDD partials (psi^2 column 0);
// lc = [Ng][2] (S_hi/dg, max(denom, eps)); lite_energy_grid(lanes) partial pairs.
template <typename T>
cudaError_t launch_lite_energy(T* F, const double* lc, double dt, int Ng, long long lanes, const double* dc, int NA,
                               int Ny, int Nz, int trap, double* partials, cudaStream_t s);
int lite_energy_grid(long long lanes);
template <typename T> cudaError_t launch_transport(const TransportArgs<T>& a, int ang_chunk, cudaStream_t s);
template <typename T> cudaError_t launch_angle(const AngleArgs<T>& a, cudaStream_t s);
template <typename T> cudaError_t launch_source_angular(const SourceArgs<T>& a, cudaStream_t s);
template <typename T> cudaError_t launch_source_energy(const SourceArgs<T>& a, int tile_e, cudaStream_t s);
template <typename T> cudaError_t launch_init_beam(T* F, const double* yza, const double* e, long long per_e,
                                                   int Ng, cudaStream_t s);

// Sum of partials [n][2] (plus column 0 of partials2 [n2][2]) into
// hist_idd[*counter] and hist_proxy[*counter], scaled by idd_scale (column 0)
// and proxy_scale (column 1 of partials only); increments the counter when
// advance != 0.  n and n2 may be 0.
cudaError_t launch_finalize_idd(const double* partials, int n, const double* partials2, int n2,
                                double idd_scale, double proxy_scale, double* hist_idd,
                                double* hist_proxy, int* counter, int capacity, int advance,
                                cudaStream_t s);
// Stand-alone IDD partials of one species (F, f) when it was not fused into
// an energy pass.  partials: [grid][2].
template <typename T>
cudaError_t launch_idd_partials(const T* F, const T* f, const double* dose_coef, int Ng, long long lanes,
                                int NA, int Ny, int Nz, int trapezoidal, int with_proxy, double* partials,
                                int grid, cudaStream_t s);
// Per-group moments (Eq. 25 diagnostics): out[2*ek] += sum psi^1, out[2*ek+1] += sum psi^2.
template <typename T>
cudaError_t launch_energy_moments(const T* F, const T* f, const T* F1, const T* f1, int Ng, long long per_e,
                                  double weight, double* out, cudaStream_t s);
template <typename Tin, typename Tout>
cudaError_t launch_convert(const Tin* in, Tout* out, long long n, cudaStream_t s);
// YZ dose plane of the current state (spot diagnostics): plane[pos], nyz values.
template <typename T>
cudaError_t launch_spot_plane(const T* F, const T* f, const T* F1, const T* f1, const double* dose_coef, int Ng,
                              int nyz, int NA, double dudv, double* plane, cudaStream_t s);

// Tensor-core (tcgen05) angular contraction of the source, float state
// (kernels_umma.cu): pack the A operand into ablob (umma_pack_bytes), then a
// bulk-copy-fed GEMM; bblob from launch_build_umma_blob with BK = 16; err receives a
// non-zero code if a CTA's bounded wait ran out.
// The epilogue writes A1 / A2 split into bf16 hi / lo into q (umma_q_bytes,
// the energy stage's operand layout); rows of groups it does not write must
// be zero.  packed (may be null) is recorded on s once the pack, the last
// reader of P1 and P2, has been enqueued.  pack = false: ablob already holds
// the operand (written by energy_fused_kernel); P1, P2 are not read.
// ulist / ubegin (may be null: every k chunk, full width): the k chunks of
// source group gz and output tile nt whose kernel block has a non-zero entry,
// entries ubegin[gz * n_ntiles + nt] .. ubegin[gz * n_ntiles + nt + 1] - 1 of
// ulist, each {k chunk, first column, columns} with the column range a
// multiple of 16 covering the chunk's non-zero columns in the tile
// (build_umma_ranges); the other chunks add nothing and are skipped.
cudaError_t launch_source_angular_pipe(const float* P1, const float* P2, uint8_t* ablob, const uint8_t* bblob,
                                       const int* groups, int n_groups, uint8_t* q, int Ng, int* err, int nyz,
                                       int NA, int NT, int BK, int n_ntiles, const int4* ulist, const int* ubegin,
                                       cudaStream_t s, cudaEvent_t packed = nullptr, bool pack = true);
// Host: the entries of ulist / ubegin from the float angular kernel kv
// ([Ng][NA in][NA out]) of the source groups.
void build_umma_ranges(const float* kv, const int* groups, int n_groups, int NA, int NT, int BK, int n_ntiles,
                       std::vector<int4>& list, std::vector<int>& begin);
size_t umma_pack_bytes(int n_groups, int nyz, int NA, int BK);
size_t umma_q_bytes(long long per_e, int Ng);
// Tensor-core energy stage: S[e][l] from q with the coefficient tiles and
// work lists of build_energy_umma (n_et = ceil(Ng / 256) output tiles).
cudaError_t launch_source_energy_umma(const uint8_t* q, const uint8_t* eblob, const int* work, const int* work_begin,
                                      int n_et, int emax_cols, float* S, int* err, long long per_e, int Ng,
                                      cudaStream_t s);
size_t energy_umma_smem(int emax_cols);
// Host: split-bf16 tiles of dg e1 and dg e2 / 3 over the bands, work items
// {chunk, first column, columns, first e group} per 256-group output tile
// (begin = offsets, in items), and the widest item.
void build_energy_umma(const double* e1, const double* e2, const int* band_begin, const int* band_end, int Ng,
                       double dg, std::vector<uint8_t>& blob, std::vector<int>& work, std::vector<int>& begin,
                       int& emax_cols);
// Split-bf16 B tiles of the float ker_v ([Ng][NA][NA], device) for the listed
// groups (device array), in the kernel's shared-memory layout, built on the
// device into blob (umma_blob_bytes bytes).
size_t umma_blob_bytes(int n_groups, int NA, int NT, int BK);
cudaError_t launch_build_umma_blob(const float* ker_v, const int* groups, int n_groups, int NA, int NT, int BK,
                                   uint8_t* blob, cudaStream_t s);

// Dynamic shared memory of one transport block (tile ty x tz, ac angles).
size_t transport_smem(int Ny1, int Nz1, int ty, int tz, int ac, size_t elem);
// Whole-plane transport for square planes of the compiled sizes
// (transport_plane_supported); ang_chunk 8 or 16 (float), 4 or 8 (double).
template <typename T> cudaError_t launch_transport_plane(const TransportArgs<T>& a, int ang_chunk, cudaStream_t s);
bool transport_plane_supported(int Ny, int Nz);
// True when NA is even and angles (2i, 2i+1) share the signs of omega_y and
// omega_z ([NA][2] table): the float whole-plane kernel may then pair them.
bool transport_pairs_ok(const double* omega, int NA);
// Float state, paired angles, square planes of the compiled sizes
// (transport_cluster_supported): one thread-block cluster per (group,
// 8-angle chunk) plane, in place.
cudaError_t launch_transport_cluster(const TransportArgs<float>& a, cudaStream_t s);
bool transport_cluster_supported(int Ny, int Nz);
// Any plane, in 27 x 27 output tiles with a 4-cell halo, out of place;
// ang_chunk 4 or 8 (float), 2 or 4 (double).
template <typename T> cudaError_t launch_transport_tiles(const TransportArgs<T>& a, int ang_chunk, cudaStream_t s);
size_t transport_tile_smem(int R, int ac, size_t elem);
size_t transport_plane_smem(int NP, int ac, size_t elem);

int energy_grid(long long lanes, int block);
int idd_partials_grid(long long lanes);

// Message that bfpn_last_error(NULL) returns on this thread, for entry points
// that take no context.
void set_context_free_error(const std::string& msg);

}  // namespace bfpn
