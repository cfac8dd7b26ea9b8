// Tensor-core (tcgen05 / UMMA) angular contraction of the catastrophic
// source, mixed precision:
//
//   A1[g, pos, out] = sum_in max(P1[g, pos, in], 0) * ker_v[g, in, out]
//   A2[g, pos, out] = sum_in P2[g, pos, in]         * ker_v[g, in, out]
//
// One CTA computes a 64-position x N_T-output tile of one source group for
// both operands at once: UMMA rows 0..63 hold max(P1, 0), rows 64..127 hold
// P2 of the same positions, and they share the B operand (ker_v).  Operands
// are split into bf16 hi + lo parts; D += Ah Bh + Ah Bl + Al Bh accumulates
// in fp32 in tensor memory (relative error ~2^-16 per product).
//
// Shared-memory operands use the UMMA K-major no-swizzle layout: 8-row x
// 16-byte core matrices, rows of a core matrix 16 B apart, core matrices
// along M/N 128 B apart (SBO) and along K one M/N-extent apart (LBO).  The B
// tiles are pre-arranged in that layout on the host (tables); a pack kernel
// writes the A tiles in it once per source evaluation; both are fetched with
// cp.async.bulk (no multicast).  Every mbarrier wait is bounded; on a timeout
// the CTA records an error code, drains what it issued (bounded), frees its
// tensor memory and returns.

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

// Byte offset of element (row, k) in a K-major no-swizzle tile of `rows`
// rows: core matrix (row/8, k/8) of 8 x 8 bf16.
__host__ __device__ inline size_t umma_kmajor_offset(int row, int k, int rows) {
    return (static_cast<size_t>(k >> 3) * (rows >> 3) + (row >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2;
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
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const float v = (row_ok && k0 + q < a.NA) ? __ldg(src + k0 + q) : 0.f;
        x[q] = is_p2 ? v : fmaxf(v, 0.f);
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
    float* A1;
    float* A2;
    int* err;
    int nyz, NA, NT, nk, n_ntiles, n_mt;
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
    const int nk = a.nk;

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

    const uint8_t* __restrict__ ablob = a.ablob + (static_cast<size_t>(gz) * a.n_mt + mt) * nk * (2 * a_part);
    const uint8_t* __restrict__ bblob =
        a.bblob + (static_cast<size_t>(gz) * a.n_ntiles + nt) * nk * static_cast<size_t>(2 * b_part);
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(NT >> 3) << 17) |
                           (static_cast<uint32_t>(kRows >> 4) << 24);

    if (tid == 0) {
        int issued[kPipe] = {}, landed[kPipe] = {}, committed[kPipe] = {}, drained[kPipe] = {};
        auto issue = [&](int it) {
            const int st = it % kPipe;
            uint8_t* sA = smem + st * stage_bytes;
            mbar_expect_tx(&bar_full[st], 2 * a_part + 2 * b_part);
            bulk_copy_g2s(sA, ablob + static_cast<size_t>(it) * 2 * a_part, 2 * a_part, &bar_full[st]);
            bulk_copy_g2s(sA + 2 * a_part, bblob + static_cast<size_t>(it) * 2 * b_part, 2 * b_part, &bar_full[st]);
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
            const uint32_t aA = smem_u32(smem + st * stage_bytes), aB = aA + 2 * a_part;
            constexpr uint32_t lboA = (kRows / 8) * 128;
            const uint32_t lboB = (NT / 8) * 128;
#pragma unroll
            for (int j = 0; j < BK / 16; ++j) {
                const uint64_t ah = umma_desc(aA + j * 2 * lboA, lboA, 128);
                const uint64_t al = umma_desc(aA + a_part + j * 2 * lboA, lboA, 128);
                const uint64_t bh = umma_desc(aB + j * 2 * lboB, lboB, 128);
                const uint64_t bl = umma_desc(aB + b_part + j * 2 * lboB, lboB, 128);
                umma_bf16(tmem, ah, bh, idesc, (it > 0 || j > 0) ? 1u : 0u);
                umma_bf16(tmem, ah, bl, idesc, 1u);
                umma_bf16(tmem, al, bh, idesc, 1u);
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
        // each thread moves 16-column slices of its accumulator row into a
        // [128][17]-float tile, then each warp writes whole rows so that every
        // store instruction covers 16 consecutive outputs of one position.
        float* tile = reinterpret_cast<float*>(smem);
        constexpr int TS = 17;  // padded row stride: conflict-free both ways
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
            // 128 rows x 16 columns: each warp instruction writes 2 rows x 16 columns
            const int half = (tid & 31) >> 4, col = tid & 15;
            const int n = n0 + c0 + col;
            for (int r = warp * 2 + half; r < kRows; r += 8) {
                const int pos = m0 + (r & (kPos - 1));
                if (pos < a.nyz && n < a.NA)
                    ((r >= kPos) ? a.A2 : a.A1)[(static_cast<size_t>(g) * a.nyz + pos) * a.NA + n] = tile[r * TS + col];
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
                                       const int* groups, int n_groups, float* A1, float* A2, int* err, int nyz,
                                       int NA, int NT, int BK, int n_ntiles, cudaStream_t s) {
    if (n_groups <= 0) return cudaSuccess;
    if (BK != 16 || NT % 16 != 0 || NT < 16 || NT > 256) return cudaErrorInvalidValue;
    const int n_mt = (nyz + kPos - 1) / kPos, nk = (NA + BK - 1) / BK;
    UmmaPackArgs p{P1, P2, groups, ablob, nyz, NA, nk, n_mt, BK};
    const long long per_group = static_cast<long long>(n_mt) * nk * kRows * (BK / 8);
    if ((per_group + 255) / 256 > 0x7fffffffLL || n_groups > 65535) return cudaErrorInvalidConfiguration;
    pack_source_operand_kernel<<<dim3(static_cast<unsigned>((per_group + 255) / 256), n_groups), 256, 0, s>>>(p);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    UmmaPipeArgs a{ablob, bblob, groups, A1, A2, err, nyz, NA, NT, nk, n_ntiles, n_mt};
    size_t smem = umma_pipe_smem(NT, BK);
    // at most two CTAs per SM when each holds 256 tensor-memory columns (512 per SM)
    if (NT > 128) smem = std::max<size_t>(smem, 80 * 1024);
    auto kern = source_angular_umma_pipe_kernel<16>;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    dim3 grid(n_ntiles, n_mt, n_groups);
    if (grid.y > 65535 || grid.z > 65535) return cudaErrorInvalidConfiguration;
    kern<<<grid, kRows, smem, s>>>(a);
    return cudaGetLastError();
}

// Host: B tiles of every used group in the device layout of the kernel above.
void build_umma_blob(const double* ker_v, const int* groups, int n_groups, int NA, int NT, int BK,
                     std::vector<uint8_t>& blob) {
    const int nk = (NA + BK - 1) / BK;
    const int n_ntiles = (NA + NT - 1) / NT;
    const size_t part = static_cast<size_t>(NT) * BK * 2;
    blob.assign(static_cast<size_t>(n_groups) * n_ntiles * nk * 2 * part, 0);
    for (int z = 0; z < n_groups; ++z) {
        const double* K = ker_v + static_cast<size_t>(groups[z]) * NA * NA;  // [in][out]
        for (int t = 0; t < n_ntiles; ++t)
            for (int kc = 0; kc < nk; ++kc) {
                uint8_t* base = blob.data() + ((static_cast<size_t>(z) * n_ntiles + t) * nk + kc) * 2 * part;
                for (int nn = 0; nn < NT; ++nn) {
                    const int n = t * NT + nn;
                    if (n >= NA) continue;
                    for (int kk = 0; kk < BK; ++kk) {
                        const int k = kc * BK + kk;
                        if (k >= NA) continue;
                        const float v = static_cast<float>(K[static_cast<size_t>(k) * NA + n]);
                        const __nv_bfloat16 h = __float2bfloat16_rn(v);
                        const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
                        const size_t off = umma_kmajor_offset(nn, kk, NT);
                        std::memcpy(base + off, &h, 2);
                        std::memcpy(base + part + off, &l, 2);
                    }
                }
            }
    }
}

}  // namespace bfpn
