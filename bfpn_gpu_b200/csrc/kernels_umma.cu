// Tensor-core (tcgen05 / UMMA) catastrophic source, mixed precision, in two
// contractions (secondarySourceFromPrimaryKernel, energy_solver.cu:287-333,
// factorised):
//
//   angular:  A1[s, pos, out] = sum_in max(P1[s, pos, in], 0) * ker_v[s, in, out]
//             A2[s, pos, out] = sum_in P2[s, pos, in]         * ker_v[s, in, out]
//   energy:   S[e, l] = sum_{s in band(e)} (dg e1[e, s]) A1[s, l] + (dg e2[e, s] / 3) A2[s, l]
//
// with l = pos * NA + out.  Operands are split into bf16 hi + lo parts;
// D += Ah Bh + Ah Bl + Al Bh accumulates in fp32 in tensor memory (relative
// error ~2^-16 per product).
//
// Angular: one CTA computes a 64-position x N_T-output tile of one source
// group for both operands at once: UMMA rows 0..63 hold max(P1, 0), rows
// 64..127 P2 of the same positions, sharing the B operand (ker_v).  Operands
// use the K-major no-swizzle layout (8-row x 16-byte core matrices); the B
// tiles are arranged on the host, a pack kernel writes the A tiles once per
// source evaluation.  The epilogue writes A1 / A2 split into bf16 hi / lo in
// the energy stage's operand layout (below), so the energy stage reads them
// with plain bulk copies.
//
// Energy: one CTA owns 128 lanes (UMMA M, the A operand, MN-major) and up to
// 256 output groups (the accumulator columns).  For every 16-group chunk of
// source groups that some output of the tile uses, it multiplies the chunk's
// 4 x 128 x 16 A tile by the coefficient tile of the outputs whose band meets
// the chunk (B operand, K-major, N = that output range rounded to 16), so
// tensor-core work follows the band.
//
// All operand moves are cp.async.bulk (no multicast).  Every mbarrier wait is
// bounded; on a timeout the CTA records an error code, drains what it issued
// (bounded), frees its tensor memory and returns.

#include "common.cuh"
#include "async_copy.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <vector>

namespace bfpn {
namespace {

constexpr int kRows = 128;       // UMMA M: 64 positions x 2 operands
constexpr int kPos = 64;
// K-major, no swizzle: start address, LBO (K direction), SBO (M/N direction), version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&v);
}

}  // namespace

// Byte offset of element (plane, s, l) in the energy stage's A operand: lanes
// in tiles of 128, source groups in rows of 8.  One (lane tile, 8 groups)
// block is 8 KB: 4 planes (A1 hi, A1 lo, A2 hi, A2 lo) x 2 atoms of 64 lanes
// x 8 rows (one per group) x 128 B, the 16-byte pieces of row r permuted to
// j ^ r -- the shared-memory image of an MN-major 128-byte-swizzled UMMA
// operand, so that a plain bulk copy of 16 groups (16 KB) lands ready to use.
// nsg = 2 * ceil(Ng / 16) group rows per lane tile.
__host__ __device__ inline size_t q_offset(int plane, int s, long long l, int nsg) {
    const long long t = l >> 7;
    const int li = static_cast<int>(l & 127), sr = s & 7;
    return ((static_cast<size_t>(t) * nsg + (s >> 3)) * 4 + plane) * 2048 + (li >> 6) * 1024 + sr * 128 +
           ((((li >> 3) & 7) ^ sr) << 4) + (li & 7) * 2;
}

size_t umma_q_bytes(long long per_e, int Ng) {
    const size_t tiles = static_cast<size_t>((per_e + 127) / 128), nsg = 2 * static_cast<size_t>((Ng + 15) / 16);
    return tiles * nsg * 8192;
}

// ---------------------------------------------------------------------------
// Pipelined form.  A pack kernel writes the A operand of every (group,
// position tile, k chunk) once, already split into bf16 hi / lo and laid out
// as the UMMA core-matrix tile (rows 0..63 max(P1, 0), rows 64..127 P2), so
// the GEMM kernel moves both operands with plain bulk copies: one thread keeps
// kPipe stages of A and B in flight, issues the MMAs of each stage as it lands
// and refills a stage as soon as the MMAs that read it have completed.  The
// other threads only wait for the final commit and run the epilogue.
// ---------------------------------------------------------------------------
constexpr int kPipe = 4;

struct UmmaPackArgs {
    const float* P1;
    const float* P2;
    const int* groups;
    uint8_t* ablob;          // [n_groups][n_mt][nk][hi|lo][128 x BK bf16, core layout]
    int nyz, NA, nk, n_mt, BK;
};

// One thread per (row, 8-value k group) of one (group, m tile, k chunk) tile.
__global__ void __launch_bounds__(256) pack_source_operand_kernel(UmmaPackArgs a) {
    const int per_tile = kRows * (a.BK / 8);
    const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;  // gridDim.y = groups
    if (idx >= static_cast<long long>(a.n_mt) * a.nk * per_tile) return;
    const int gz = blockIdx.y;
    const int r8 = static_cast<int>(idx % per_tile);
    const long long tile = idx / per_tile;  // mt * nk + kc
    const int kc = static_cast<int>(tile % a.nk), mt = static_cast<int>(tile / a.nk);
    const int row = r8 / (a.BK / 8), c = r8 % (a.BK / 8);
    const int pos = mt * kPos + (row & (kPos - 1));
    const bool is_p2 = row >= kPos;
    const int k0 = kc * a.BK + c * 8;
    float x[8], r[8];
    const int g = a.groups[gz];
    const float* __restrict__ src = (is_p2 ? a.P2 : a.P1) + (static_cast<size_t>(g) * a.nyz + pos) * a.NA;
    const bool row_ok = pos < a.nyz;
    if (row_ok && (a.NA & 3) == 0 && k0 + 8 <= a.NA) {  // two 16-byte loads (row starts are 16-byte aligned)
        const float4 u = __ldg(reinterpret_cast<const float4*>(src + k0));
        const float4 w = __ldg(reinterpret_cast<const float4*>(src + k0 + 4));
        x[0] = u.x; x[1] = u.y; x[2] = u.z; x[3] = u.w;
        x[4] = w.x; x[5] = w.y; x[6] = w.z; x[7] = w.w;
    } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) x[q] = (row_ok && k0 + q < a.NA) ? __ldg(src + k0 + q) : 0.f;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        if (!is_p2) x[q] = fmaxf(x[q], 0.f);
        r[q] = x[q] - __bfloat162float(__float2bfloat16_rn(x[q]));
    }
    uint4 hi, lo;
    hi.x = pack_bf16(x[0], x[1]);
    hi.y = pack_bf16(x[2], x[3]);
    hi.z = pack_bf16(x[4], x[5]);
    hi.w = pack_bf16(x[6], x[7]);
    lo.x = pack_bf16(r[0], r[1]);
    lo.y = pack_bf16(r[2], r[3]);
    lo.z = pack_bf16(r[4], r[5]);
    lo.w = pack_bf16(r[6], r[7]);
    const size_t a_part = static_cast<size_t>(kRows) * a.BK * 2;
    uint8_t* base = a.ablob + ((static_cast<size_t>(gz) * a.n_mt + mt) * a.nk + kc) * 2 * a_part;
    const size_t off = umma_kmajor_offset(row, c * 8, kRows);
    *reinterpret_cast<uint4*>(base + off) = hi;
    *reinterpret_cast<uint4*>(base + a_part + off) = lo;
}

struct UmmaPipeArgs {
    const uint8_t* ablob;
    const uint8_t* bblob;    // [n_groups][n_ntiles][nk][hi|lo][N_T x BK bf16, core layout]
    const int* groups;
    uint8_t* q;              // energy-stage operand (q_offset layout)
    int* err;
    const int4* ulist;       // non-zero k chunks and column ranges (or null: all, full width)
    const int* ubegin;
    int nyz, NA, NT, nk, n_ntiles, n_mt, nsg;
};

template <int BK>
__global__ void __launch_bounds__(128, 1) source_angular_umma_pipe_kernel(UmmaPipeArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar_full[kPipe];
    __shared__ __align__(8) uint64_t bar_mma[kPipe];
    __shared__ uint32_t tmem_base_slot;
    __shared__ int fail_flag;

    const int NT = a.NT;
    constexpr uint32_t a_part = kRows * BK * 2;
    const uint32_t b_part = NT * BK * 2;
    const uint32_t stage_bytes = 2 * a_part + 2 * b_part;
    const int nt = blockIdx.x, mt = blockIdx.y, gz = blockIdx.z;
    const int g = a.groups[gz];
    const int m0 = mt * kPos, n0 = nt * NT;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t ncols = NT <= 32 ? 32 : NT <= 64 ? 64 : NT <= 128 ? 128 : 256;
    // the k chunks this tile multiplies: the non-zero ones of its kernel block
    const int u0 = a.ulist ? __ldg(a.ubegin + gz * a.n_ntiles + nt) : 0;
    const int nk = a.ulist ? __ldg(a.ubegin + gz * a.n_ntiles + nt + 1) - u0 : a.nk;
    auto entry = [&](int it) {
        return a.ulist ? __ldg(a.ulist + u0 + it) : make_int4(it, 0, NT, 0);
    };

    if (tid == 0) {
        for (int s = 0; s < kPipe; ++s) {
            mbar_init(&bar_full[s], 1);
            mbar_init(&bar_mma[s], 1);
        }
        mbar_init_fence();
        fail_flag = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_slot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_slot;
    {
        // zero the accumulator: the MMAs cover only the columns their chunks reach
        const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
        const uint32_t z = 0;
        for (uint32_t c0 = 0; c0 < ncols; c0 += 16)
            asm volatile(
                "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};" ::"r"(
                    tmem + lane_base + c0),
                "r"(z)
                : "memory");
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    const uint8_t* __restrict__ ablob = a.ablob + (static_cast<size_t>(gz) * a.n_mt + mt) * a.nk * (2 * a_part);
    const uint8_t* __restrict__ bblob =
        a.bblob + (static_cast<size_t>(gz) * a.n_ntiles + nt) * a.nk * static_cast<size_t>(2 * b_part);
    const uint32_t idesc0 = (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(kRows >> 4) << 24);

    if (tid == 0) {
        int issued[kPipe] = {}, landed[kPipe] = {}, committed[kPipe] = {}, drained[kPipe] = {};
        auto issue = [&](int it) {
            const int st = it % kPipe;
            const int kc = entry(it).x;
            uint8_t* sA = smem + st * stage_bytes;
            mbar_expect_tx(&bar_full[st], 2 * a_part + 2 * b_part);
            bulk_copy_g2s(sA, ablob + static_cast<size_t>(kc) * 2 * a_part, 2 * a_part, &bar_full[st]);
            bulk_copy_g2s(sA + 2 * a_part, bblob + static_cast<size_t>(kc) * 2 * b_part, 2 * b_part, &bar_full[st]);
            ++issued[st];
        };
        bool bad = false;
        for (int it = 0; it < min(kPipe, nk); ++it) issue(it);
        for (int it = 0; it < nk && !bad; ++it) {
            const int st = it % kPipe;
            if (!mbar_wait(&bar_full[st], (it / kPipe) & 1)) {
                bad = true;
                break;
            }
            ++landed[st];
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int4 en = entry(it);  // {k chunk, first column, columns}
            const uint32_t aA = smem_u32(smem + st * stage_bytes), aB = aA + 2 * a_part + (en.y / 8) * 128;
            constexpr uint32_t lboA = (kRows / 8) * 128;
            const uint32_t lboB = (NT / 8) * 128;
            const uint32_t idesc = idesc0 | (static_cast<uint32_t>(en.z >> 3) << 17);
            const uint32_t dcol = tmem + static_cast<uint32_t>(en.y);
#pragma unroll
            for (int j = 0; j < BK / 16; ++j) {
                const uint64_t ah = umma_desc(aA + j * 2 * lboA, lboA, 128);
                const uint64_t al = umma_desc(aA + a_part + j * 2 * lboA, lboA, 128);
                const uint64_t bh = umma_desc(aB + j * 2 * lboB, lboB, 128);
                const uint64_t bl = umma_desc(aB + b_part + j * 2 * lboB, lboB, 128);
                umma_bf16(dcol, ah, bh, idesc, 1u);
                umma_bf16(dcol, ah, bl, idesc, 1u);
                umma_bf16(dcol, al, bh, idesc, 1u);
            }
            umma_commit(&bar_mma[st]);
            ++committed[st];
            // refill the stage of the previous iteration once its MMAs are done
            // (this iteration's MMAs stay queued meanwhile)
            const int prev = it - 1;
            if (prev >= 0 && prev + kPipe < nk) {
                const int ps = prev % kPipe;
                if (!mbar_wait(&bar_mma[ps], (prev / kPipe) & 1)) {
                    bad = true;
                    break;
                }
                ++drained[ps];
                issue(prev + kPipe);
            }
        }
        // the last commit covers every MMA issued before it
        if (!bad && nk > 0) {
            const int last = nk - 1;
            if (!mbar_wait(&bar_mma[last % kPipe], (last / kPipe) & 1)) bad = true;
        }
        if (bad) {
            atomicExch(a.err, 1);
            // drain what was issued: the last commit and any copy not seen to land
            for (int s = 0; s < kPipe; ++s) {
                if (committed[s] > drained[s]) mbar_wait(&bar_mma[s], (committed[s] - 1) & 1);
                if (issued[s] > landed[s]) mbar_wait(&bar_full[s], (issued[s] - 1) & 1);
            }
            fail_flag = 1;
        }
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!fail_flag) {
        // Epilogue through shared memory (the pipeline buffers are free now):
        // 16-column slices of the accumulator go to a [128][17]-float tile;
        // then each thread takes 8 consecutive outputs of one row, splits
        // them into bf16 hi / lo and writes both into the energy operand
        // layout.  Two threads share a row, so with 8-aligned lanes one warp
        // store covers whole 32-byte pieces.
        float* tile = reinterpret_cast<float*>(smem);
        constexpr int TS = 17;  // padded row stride
        const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
        for (int c0 = 0; c0 < NT; c0 += 16) {
            uint32_t v[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(tmem + lane_base + c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 16; ++q) tile[tid * TS + q] = __uint_as_float(v[q]);
            __syncthreads();
            for (int task = tid; task < 2 * kRows; task += 128) {
                const int r = task >> 1, h = task & 1;
                const int pos = m0 + (r & (kPos - 1));
                const int n = n0 + c0 + 8 * h;
                if (pos >= a.nyz || n >= a.NA) continue;
                const int plane = r >= kPos ? 2 : 0;
                const long long l = static_cast<long long>(pos) * a.NA + n;
                const float* x = tile + r * TS + 8 * h;
                if ((l & 7) == 0 && n + 8 <= a.NA) {
                    float y[8], z[8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        y[k] = x[k];
                        z[k] = y[k] - __bfloat162float(__float2bfloat16_rn(y[k]));
                    }
                    const uint4 hi = make_uint4(pack_bf16(y[0], y[1]), pack_bf16(y[2], y[3]), pack_bf16(y[4], y[5]),
                                                pack_bf16(y[6], y[7]));
                    const uint4 lo = make_uint4(pack_bf16(z[0], z[1]), pack_bf16(z[2], z[3]), pack_bf16(z[4], z[5]),
                                                pack_bf16(z[6], z[7]));
                    *reinterpret_cast<uint4*>(a.q + q_offset(plane, g, l, a.nsg)) = hi;
                    *reinterpret_cast<uint4*>(a.q + q_offset(plane + 1, g, l, a.nsg)) = lo;
                } else {
                    for (int k = 0; k < 8 && n + k < a.NA; ++k) {
                        const __nv_bfloat16 hb = __float2bfloat16_rn(x[k]);
                        const __nv_bfloat16 lb = __float2bfloat16_rn(x[k] - __bfloat162float(hb));
                        *reinterpret_cast<__nv_bfloat16*>(a.q + q_offset(plane, g, l + k, a.nsg)) = hb;
                        *reinterpret_cast<__nv_bfloat16*>(a.q + q_offset(plane + 1, g, l + k, a.nsg)) = lb;
                    }
                }
            }
            __syncthreads();
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
    }
}

size_t umma_pack_bytes(int n_groups, int nyz, int NA, int BK) {
    const size_t n_mt = (nyz + kPos - 1) / kPos, nk = (NA + BK - 1) / BK;
    return static_cast<size_t>(n_groups) * n_mt * nk * 2 * kRows * BK * 2;
}

size_t umma_pipe_smem(int NT, int BK) {
    return static_cast<size_t>(kPipe) * (2 * static_cast<size_t>(kRows) * BK * 2 + 2 * static_cast<size_t>(NT) * BK * 2);
}

cudaError_t launch_source_angular_pipe(const float* P1, const float* P2, uint8_t* ablob, const uint8_t* bblob,
                                       const int* groups, int n_groups, uint8_t* q, int Ng, int* err, int nyz,
                                       int NA, int NT, int BK, int n_ntiles, const int4* ulist, const int* ubegin,
                                       cudaStream_t s, cudaEvent_t packed, bool pack) {
    if (n_groups <= 0) return packed ? cudaEventRecord(packed, s) : cudaSuccess;
    if (BK != 16 || NT % 16 != 0 || NT < 16 || NT > 256) return cudaErrorInvalidValue;
    const int n_mt = (nyz + kPos - 1) / kPos, nk = (NA + BK - 1) / BK;
    cudaError_t e = cudaSuccess;
    if (pack) {
        UmmaPackArgs p{P1, P2, groups, ablob, nyz, NA, nk, n_mt, BK};
        const long long per_group = static_cast<long long>(n_mt) * nk * kRows * (BK / 8);
        if ((per_group + 255) / 256 > 0x7fffffffLL || n_groups > 65535) return cudaErrorInvalidConfiguration;
        pack_source_operand_kernel<<<dim3(static_cast<unsigned>((per_group + 255) / 256), n_groups), 256, 0, s>>>(p);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (packed && (e = cudaEventRecord(packed, s)) != cudaSuccess) return e;
    UmmaPipeArgs a{ablob, bblob, groups, q, err, ulist, ubegin, nyz, NA, NT, nk, n_ntiles, n_mt, 2 * ((Ng + 15) / 16)};
    size_t smem = umma_pipe_smem(NT, BK);
    // at most two CTAs per SM when each holds 256 tensor-memory columns (512 per SM)
    if (NT > 128) smem = std::max<size_t>(smem, 80 * 1024);
    auto kern = source_angular_umma_pipe_kernel<16>;
    e = allow_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
    if (e != cudaSuccess) return e;
    dim3 grid(n_ntiles, n_mt, n_groups);
    if (grid.y > 65535 || grid.z > 65535) return cudaErrorInvalidConfiguration;
    kern<<<grid, kRows, smem, s>>>(a);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Energy stage.  CTA (lane tile lt, output tile et) owns lanes 128 lt ..
// 128 lt + 127 (UMMA rows) and output groups 256 et .. 256 et + 255 (tensor
// memory columns, zeroed first).  Its work list holds, per 16-group source
// chunk c that some of its outputs use, the output column range [col,
// col + ncols) whose bands meet the chunk.  Per item one thread lands the
// chunk's 16 KB A tile (q_offset layout, MN-major, 128-byte swizzle) and the
// range's coefficient tile (K-major, no swizzle) with two bulk copies and
// issues 6 MMAs (hi/lo splits of both operands, A1 and A2) into that column
// range; kPipeE stages in flight.  The epilogue streams each accumulator row
// (one lane) column by column to S, 128 consecutive lanes per warp store.
// ---------------------------------------------------------------------------
constexpr int kEnergyCols = 256;
constexpr int kMaxStagesE = 4;
constexpr uint32_t kQStage = 16384;  // 16 groups x 128 lanes x 4 planes x 2 B

struct EnergyUmmaArgs {
    const uint8_t* q;
    const uint8_t* eblob;     // [chunk][e group of 8][4 planes][2 k halves][8 rows][16 B]
    const int4* work;         // {chunk, first column, columns, first e group}
    const int* work_begin;    // [n_et + 1]
    float* S;
    int* err;
    long long per_e;
    int Ng, n_et, nsg, n_eg, nst;
    uint32_t stage_bytes;
};

__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return umma_desc(addr, lbo, sbo) | (2ull << 61);
}

__global__ void __launch_bounds__(128, 1) source_energy_umma_kernel(EnergyUmmaArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar_full[kMaxStagesE];
    __shared__ __align__(8) uint64_t bar_mma[kMaxStagesE];
    __shared__ uint32_t tmem_base_slot;
    __shared__ int fail_flag;

    const int tid = threadIdx.x, warp = tid >> 5;
    const int et = static_cast<int>(blockIdx.x % a.n_et);
    const long long lt = blockIdx.x / a.n_et;
    const int w0 = a.work_begin[et], nw = a.work_begin[et + 1] - w0;
    const int nst = a.nst;
    // 128-byte swizzle atoms want 1024-byte aligned stages
    const uint32_t raw = smem_u32(smem);
    uint8_t* stages = smem + (((raw + 1023u) & ~1023u) - raw);

    if (tid == 0) {
        for (int st = 0; st < nst; ++st) {
            mbar_init(&bar_full[st], 1);
            mbar_init(&bar_mma[st], 1);
        }
        mbar_init_fence();
        fail_flag = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_slot)),
                     "r"(kEnergyCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_slot;
    const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
    {  // zero the accumulator: the MMAs of an item only add into its column range
        const uint32_t z = 0;
        for (int c0 = 0; c0 < kEnergyCols; c0 += 16)
            asm volatile(
                "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};" ::"r"(
                    tmem + lane_base + c0),
                "r"(z)
                : "memory");
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (tid == 0 && nw > 0) {
        int issued[kMaxStagesE] = {}, landed[kMaxStagesE] = {}, committed[kMaxStagesE] = {},
            drained[kMaxStagesE] = {};
        const uint8_t* __restrict__ qtile = a.q + static_cast<size_t>(lt) * a.nsg * 8192;
        auto issue = [&](int it) {
            const int st = it % nst;
            const int4 w = a.work[w0 + it];
            uint8_t* sQ = stages + st * a.stage_bytes;
            const uint32_t ebytes = static_cast<uint32_t>(w.z) * 128u;  // columns x 4 planes x 16 groups x 2 B
            mbar_expect_tx(&bar_full[st], kQStage + ebytes);
            bulk_copy_g2s(sQ, qtile + static_cast<size_t>(2 * w.x) * 8192, kQStage, &bar_full[st]);
            bulk_copy_g2s(sQ + kQStage, a.eblob + (static_cast<size_t>(w.x) * a.n_eg + w.w) * 1024, ebytes,
                          &bar_full[st]);
            ++issued[st];
        };
        constexpr uint32_t idesc_base = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) |
                                        (static_cast<uint32_t>(128 >> 4) << 24);  // f32 += bf16 x bf16, A MN-major
        bool bad = false;
        for (int it = 0; it < min(nst, nw); ++it) issue(it);
        for (int it = 0; it < nw && !bad; ++it) {
            const int st = it % nst;
            if (!mbar_wait(&bar_full[st], (it / nst) & 1)) {
                bad = true;
                break;
            }
            ++landed[st];
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int4 w = a.work[w0 + it];
            const uint32_t aQ = smem_u32(stages + st * a.stage_bytes), aE = aQ + kQStage;
            const uint32_t idesc = idesc_base | (static_cast<uint32_t>(w.z >> 3) << 17);
            const uint32_t d = tmem + static_cast<uint32_t>(w.y);
#pragma unroll
            for (int x = 0; x < 2; ++x) {  // A1 with dg e1, A2 with dg e2 / 3
                const uint64_t qh = umma_desc_sw128(aQ + (2 * x) * 2048, 1024, 8192);
                const uint64_t ql = umma_desc_sw128(aQ + (2 * x + 1) * 2048, 1024, 8192);
                const uint64_t eh = umma_desc(aE + (2 * x) * 256, 128, 1024);
                const uint64_t el = umma_desc(aE + (2 * x + 1) * 256, 128, 1024);
                umma_bf16(d, qh, eh, idesc, 1u);
                umma_bf16(d, ql, eh, idesc, 1u);
                umma_bf16(d, qh, el, idesc, 1u);
            }
            umma_commit(&bar_mma[st]);
            ++committed[st];
            const int prev = it - 1;
            if (prev >= 0 && prev + nst < nw) {
                const int ps = prev % nst;
                if (!mbar_wait(&bar_mma[ps], (prev / nst) & 1)) {
                    bad = true;
                    break;
                }
                ++drained[ps];
                issue(prev + nst);
            }
        }
        if (!bad) {
            const int last = nw - 1;
            if (!mbar_wait(&bar_mma[last % nst], (last / nst) & 1)) bad = true;
        }
        if (bad) {
            atomicExch(a.err, 2);
            for (int st = 0; st < nst; ++st) {
                if (committed[st] > drained[st]) mbar_wait(&bar_mma[st], (committed[st] - 1) & 1);
                if (issued[st] > landed[st]) mbar_wait(&bar_full[st], (issued[st] - 1) & 1);
            }
            fail_flag = 1;
        }
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!fail_flag) {
        const int E0 = et * kEnergyCols;
        const int ncol = min(kEnergyCols, a.Ng - E0);
        const long long l = lt * 128 + tid;  // accumulator row tid = lane tid of the tile
        float* __restrict__ S = a.S + static_cast<size_t>(E0) * a.per_e + l;
        for (int c0 = 0; c0 < ncol; c0 += 16) {
            uint32_t v[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(tmem + lane_base + c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (l < a.per_e) {
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    if (c0 + j < ncol) S[static_cast<size_t>(c0 + j) * a.per_e] = __uint_as_float(v[j]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kEnergyCols)
                     : "memory");
    }
}

// Stages per CTA: as many (up to 4) as keep two CTAs on an SM.
static int energy_umma_stages(int emax_cols, uint32_t* stage_bytes) {
    *stage_bytes = kQStage + static_cast<uint32_t>(emax_cols) * 128u;
    int nst = kMaxStagesE;
    while (nst > 2 && nst * static_cast<size_t>(*stage_bytes) + 1024 > 110 * 1024) --nst;
    return nst;
}

// At least 80 KB, so that no third CTA waits on an SM for tensor memory
// (two CTAs x 256 columns fill it).
size_t energy_umma_smem(int emax_cols) {
    uint32_t sb = 0;
    const int nst = energy_umma_stages(emax_cols, &sb);
    return std::max<size_t>(nst * static_cast<size_t>(sb) + 1024, 80 * 1024);
}

cudaError_t launch_source_energy_umma(const uint8_t* q, const uint8_t* eblob, const int* work, const int* work_begin,
                                      int n_et, int emax_cols, float* S, int* err, long long per_e, int Ng,
                                      cudaStream_t s) {
    if (emax_cols < 0 || emax_cols > kEnergyCols || emax_cols % 16 != 0) return cudaErrorInvalidValue;
    if (n_et != (Ng + kEnergyCols - 1) / kEnergyCols) return cudaErrorInvalidValue;
    const long long n_lt = (per_e + 127) / 128;
    if (n_lt * n_et > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    EnergyUmmaArgs a;
    a.q = q;
    a.eblob = eblob;
    a.work = reinterpret_cast<const int4*>(work);
    a.work_begin = work_begin;
    a.S = S;
    a.err = err;
    a.per_e = per_e;
    a.Ng = Ng;
    a.n_et = n_et;
    a.nsg = 2 * ((Ng + 15) / 16);
    a.n_eg = a.nsg;
    a.nst = energy_umma_stages(emax_cols, &a.stage_bytes);
    const size_t smem = energy_umma_smem(emax_cols);
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void*>(source_energy_umma_kernel), smem);
    if (e != cudaSuccess) return e;
    source_energy_umma_kernel<<<static_cast<unsigned>(n_lt * n_et), 128, smem, s>>>(a);
    return cudaGetLastError();
}

// Host: the energy stage's coefficient tiles and work lists.  Tile (chunk c,
// e group g) = 1 KB: planes dg e1 hi, dg e1 lo, dg e2 / 3 hi, dg e2 / 3 lo,
// each [2 k halves][8 outputs][8 source groups] bf16 (K-major core matrices).
void build_energy_umma(const double* e1, const double* e2, const int* band_begin, const int* band_end, int Ng,
                       double dg, std::vector<uint8_t>& blob, std::vector<int>& work, std::vector<int>& begin,
                       int& emax_cols) {
    const int nchunk = (Ng + 15) / 16, n_eg = 2 * nchunk, n_et = (Ng + kEnergyCols - 1) / kEnergyCols;
    blob.assign(static_cast<size_t>(nchunk) * n_eg * 1024, 0);
    for (int e = 0; e < Ng; ++e)
        for (int sg = band_begin[e]; sg < band_end[e]; ++sg) {
            const double v[2] = {dg * e1[static_cast<size_t>(e) * Ng + sg], dg * e2[static_cast<size_t>(e) * Ng + sg] / 3.0};
            const int c = sg >> 4, k = sg & 15;
            for (int x = 0; x < 2; ++x) {
                const float f = static_cast<float>(v[x]);
                const __nv_bfloat16 h = __float2bfloat16_rn(f);
                const __nv_bfloat16 l = __float2bfloat16_rn(f - __bfloat162float(h));
                const size_t off = ((static_cast<size_t>(c) * n_eg + (e >> 3)) * 4 + 2 * x) * 256 + (k >> 3) * 128 +
                                   (e & 7) * 16 + (k & 7) * 2;
                std::memcpy(blob.data() + off, &h, 2);
                std::memcpy(blob.data() + off + 256, &l, 2);
            }
        }
    work.clear();
    begin.assign(n_et + 1, 0);
    emax_cols = 0;
    for (int et = 0; et < n_et; ++et) {
        const int E0 = et * kEnergyCols, E1 = std::min(Ng, E0 + kEnergyCols);
        for (int c = 0; c < nchunk; ++c) {
            int lo = E1, hi = E0;
            for (int e = E0; e < E1; ++e)
                if (band_begin[e] < band_end[e] && band_begin[e] < 16 * c + 16 && band_end[e] > 16 * c) {
                    lo = std::min(lo, e);
                    hi = std::max(hi, e + 1);
                }
            if (lo >= hi) continue;
            const int col = (lo - E0) / 16 * 16, ncols = (hi - E0 + 15) / 16 * 16 - col;
            work.insert(work.end(), {c, col, ncols, (E0 + col) / 8});
            emax_cols = std::max(emax_cols, ncols);
        }
        begin[et + 1] = static_cast<int>(work.size() / 4);
    }
}

// B tiles of every used group in the device layout of the kernel above, built
// on the device from the float copy of ker_v ([Ng][NA][NA], [src][in][out]):
// one thread per 8-value k piece of one row n of one (group, n tile, k chunk)
// tile writes the piece's bf16 hi and lo halves (16 bytes each); pieces past
// NA are zeros.  Adjacent threads take adjacent rows, so the reads of ker_v
// (consecutive n) coalesce.
__global__ void build_umma_blob_kernel(const float* __restrict__ ker_v, const int* __restrict__ groups, int NA,
                                       int NT, int BK, int n_ntiles, int nk, long long n_pieces,
                                       uint8_t* __restrict__ blob) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n_pieces) return;
    const int kp = BK / 8;
    const int nn = static_cast<int>(i % NT);
    long long r = i / NT;
    const int kh = static_cast<int>(r % kp);
    r /= kp;
    const int kc = static_cast<int>(r % nk);
    r /= nk;
    const int t = static_cast<int>(r % n_ntiles);
    const int z = static_cast<int>(r / n_ntiles);
    const size_t part = static_cast<size_t>(NT) * BK * 2;
    uint8_t* base = blob + ((static_cast<size_t>(z) * n_ntiles + t) * nk + kc) * 2 * part;
    const int n = t * NT + nn, k0 = kc * BK + kh * 8;
    const float* K = ker_v + static_cast<size_t>(groups[z]) * NA * NA;
    uint32_t hw[4], lw[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        __nv_bfloat16 h2[2], l2[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int k = k0 + 2 * q + e;
            const float v = (n < NA && k < NA) ? K[static_cast<size_t>(k) * NA + n] : 0.f;
            h2[e] = __float2bfloat16_rn(v);
            l2[e] = __float2bfloat16_rn(v - __bfloat162float(h2[e]));
        }
        hw[q] = static_cast<uint32_t>(__bfloat16_as_ushort(h2[0])) |
                (static_cast<uint32_t>(__bfloat16_as_ushort(h2[1])) << 16);
        lw[q] = static_cast<uint32_t>(__bfloat16_as_ushort(l2[0])) |
                (static_cast<uint32_t>(__bfloat16_as_ushort(l2[1])) << 16);
    }
    const size_t off = umma_kmajor_offset(nn, kh * 8, NT);
    *reinterpret_cast<uint4*>(base + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    *reinterpret_cast<uint4*>(base + part + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
}

void build_umma_ranges(const float* kv, const int* groups, int n_groups, int NA, int NT, int BK, int n_ntiles,
                       std::vector<int4>& list, std::vector<int>& begin) {
    const int nk = (NA + BK - 1) / BK;
    list.clear();
    begin.assign(static_cast<size_t>(n_groups) * n_ntiles + 1, 0);
    for (int gz = 0; gz < n_groups; ++gz) {
        const float* K = kv + static_cast<size_t>(groups[gz]) * NA * NA;  // [in][out]
        for (int nt = 0; nt < n_ntiles; ++nt) {
            begin[static_cast<size_t>(gz) * n_ntiles + nt] = static_cast<int>(list.size());
            const int n0 = nt * NT, n1 = std::min(NA, n0 + NT);
            for (int kc = 0; kc < nk; ++kc) {
                int lo = NT, hi = 0;
                for (int in = kc * BK; in < std::min(NA, (kc + 1) * BK); ++in) {
                    const float* row = K + static_cast<size_t>(in) * NA;
                    for (int o = n0; o < n1; ++o)
                        if (row[o] != 0.0f) {
                            lo = std::min(lo, o - n0);
                            hi = std::max(hi, o - n0 + 1);
                        }
                }
                if (hi <= lo) continue;
                lo = lo / 16 * 16;
                hi = std::min(NT, (hi + 15) / 16 * 16);
                list.push_back(make_int4(kc, lo, hi - lo, 0));
            }
        }
    }
    begin.back() = static_cast<int>(list.size());
}

size_t umma_blob_bytes(int n_groups, int NA, int NT, int BK) {
    const size_t nk = (NA + BK - 1) / BK, n_ntiles = (NA + NT - 1) / NT;
    return static_cast<size_t>(n_groups) * n_ntiles * nk * 2 * static_cast<size_t>(NT) * BK * 2;
}

cudaError_t launch_build_umma_blob(const float* ker_v, const int* groups, int n_groups, int NA, int NT, int BK,
                                   uint8_t* blob, cudaStream_t s) {
    if (n_groups <= 0) return cudaSuccess;
    if (BK % 8 != 0 || NT % 8 != 0) return cudaErrorInvalidValue;
    const int nk = (NA + BK - 1) / BK, n_ntiles = (NA + NT - 1) / NT;
    const long long n_pieces = static_cast<long long>(n_groups) * n_ntiles * nk * (BK / 8) * NT;
    const long long grid = (n_pieces + 255) / 256;
    if (grid > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    build_umma_blob_kernel<<<static_cast<unsigned>(grid), 256, 0, s>>>(ker_v, groups, NA, NT, BK, n_ntiles, nk,
                                                                       n_pieces, blob);
    return cudaGetLastError();
}

}  // namespace bfpn
