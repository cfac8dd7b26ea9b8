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
// tiles are pre-arranged in that layout on the host (tables) and fetched
// with cp.async.bulk (no multicast); A is converted from the fp32 state by
// the CTA's threads.  Two pipeline stages: the MMAs of one stage overlap the
// conversion and copy of the next.  Every mbarrier wait is bounded; on a
// timeout the CTA records an error code, drains what it issued (bounded),
// frees its tensor memory and returns.

#include "common.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <vector>

namespace bfpn {
namespace {

constexpr int kRows = 128;       // UMMA M: 64 positions x 2 operands
constexpr int kPos = 64;
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bounded parity wait; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
    for (uint32_t i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

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

struct UmmaSourceArgs {
    const float* P1;
    const float* P2;
    const uint8_t* bblob;    // [n_groups][n_ntiles][nk][hi|lo][N_T x BK bf16, core layout]
    const int* groups;
    float* A1;
    float* A2;
    int* err;                // error word (0 = ok)
    int nyz, NA, NT, nk, n_ntiles;
};

template <int BK>
__global__ void __launch_bounds__(128, 1) source_angular_umma_kernel(UmmaSourceArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar_b[2];
    __shared__ __align__(8) uint64_t bar_mma[2];
    __shared__ uint32_t tmem_base_slot;

    const int NT = a.NT;
    const uint32_t a_part = kRows * BK * 2;       // bytes of one A part (hi or lo)
    const uint32_t b_part = NT * BK * 2;          // bytes of one B part
    const uint32_t stage_bytes = 2 * a_part + 2 * b_part;
    const int nt = blockIdx.x, mt = blockIdx.y, gz = blockIdx.z;
    const int g = a.groups[gz];
    const int m0 = mt * kPos, n0 = nt * NT;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t ncols = NT <= 32 ? 32 : NT <= 64 ? 64 : NT <= 128 ? 128 : 256;

    if (tid == 0) {
        mbar_init(&bar_b[0], 1);
        mbar_init(&bar_b[1], 1);
        mbar_init(&bar_mma[0], 1);
        mbar_init(&bar_mma[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
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

    // row of this thread in the A operand
    const int row = tid;
    const int pos = m0 + (row & (kPos - 1));
    const bool is_p2 = row >= kPos;
    const float* __restrict__ src = (is_p2 ? a.P2 : a.P1) + (static_cast<size_t>(g) * a.nyz + pos) * a.NA;
    const bool row_ok = pos < a.nyz;
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(NT >> 3) << 17) |
                           (static_cast<uint32_t>(kRows >> 4) << 24);
    const uint8_t* __restrict__ blob =
        a.bblob + (static_cast<size_t>(gz) * a.n_ntiles + nt) * a.nk * static_cast<size_t>(2 * b_part);

    // this thread's row for one stage: BK values, loaded one stage ahead of use
    const bool vec = (a.NA % 4) == 0;
    float xa[BK];
    auto load_row = [&](int k0) {
        if (vec && row_ok && k0 + BK <= a.NA) {
#pragma unroll
            for (int c = 0; c < BK / 4; ++c) {
                const float4 v = __ldg(reinterpret_cast<const float4*>(src + k0) + c);
                xa[4 * c] = v.x;
                xa[4 * c + 1] = v.y;
                xa[4 * c + 2] = v.z;
                xa[4 * c + 3] = v.w;
            }
        } else {
#pragma unroll
            for (int q = 0; q < BK; ++q) xa[q] = (row_ok && k0 + q < a.NA) ? __ldg(src + k0 + q) : 0.f;
        }
    };
    load_row(0);

    bool failed = false;
    int commits[2] = {0, 0};   // MMA commits per stage (thread 0)
    int copies[2] = {0, 0};    // B copies issued per stage (thread 0)
    int copies_seen[2] = {0, 0};
    for (int it = 0; it < a.nk; ++it) {
        const int st = it & 1;
        uint8_t* sA = smem + st * stage_bytes;
        uint8_t* sB = sA + 2 * a_part;
        if (it >= 2) {  // the MMAs that read this stage two iterations ago are done
            const bool ok = mbar_wait(&bar_mma[st], ((it - 2) >> 1) & 1);
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
        }
        if (tid == 0) {
            mbar_expect_tx(&bar_b[st], 2 * b_part);
            bulk_copy_g2s(sB, blob + static_cast<size_t>(it) * 2 * b_part, 2 * b_part, &bar_b[st]);
            ++copies[st];
        }
        // A: split the prefetched row into hi / lo bf16, core-matrix layout
#pragma unroll
        for (int c = 0; c < BK / 8; ++c) {
            float x[8], r[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                x[q] = is_p2 ? xa[c * 8 + q] : fmaxf(xa[c * 8 + q], 0.f);
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
            const size_t off = umma_kmajor_offset(row, c * 8, kRows);
            *reinterpret_cast<uint4*>(sA + off) = hi;
            *reinterpret_cast<uint4*>(sA + a_part + off) = lo;
        }
        if (it + 1 < a.nk) load_row((it + 1) * BK);  // in flight while this stage's MMAs run
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        bool bad = false;
        if (tid == 0) {
            if (!mbar_wait(&bar_b[st], (it >> 1) & 1)) {
                bad = true;
            } else {
                ++copies_seen[st];
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t aA = smem_u32(sA), aB = smem_u32(sB);
                const uint32_t lboA = (kRows / 8) * 128, lboB = (NT / 8) * 128;
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
                ++commits[st];
            }
        }
        if (__syncthreads_or(bad)) {
            failed = true;
            break;
        }
    }
    // wait for the last commit (it covers every MMA issued before it)
    if (!failed && a.nk > 0) {
        const int last = a.nk - 1;
        const bool ok = mbar_wait(&bar_mma[last & 1], (last >> 1) & 1);
        failed = __syncthreads_or(!ok);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!failed) {
        float* __restrict__ dst = (is_p2 ? a.A2 : a.A1) + (static_cast<size_t>(g) * a.nyz + pos) * a.NA;
        const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
        for (int c0 = 0; c0 < NT; c0 += 16) {
            uint32_t v[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(tmem + lane_base + c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row_ok) {
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const int n = n0 + c0 + q;
                    if (n < a.NA) dst[n] = __uint_as_float(v[q]);
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(a.err, 1);
        // drain what this CTA issued, each wait bounded: the last commit of
        // each stage, and any copy whose completion was not observed
        for (int s2 = 0; s2 < 2; ++s2) {
            if (commits[s2] > 0) mbar_wait(&bar_mma[s2], (commits[s2] - 1) & 1);
            if (copies[s2] > copies_seen[s2]) mbar_wait(&bar_b[s2], (copies[s2] - 1) & 1);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
    }
}

size_t umma_source_smem(int NT, int BK) { return 2 * (2 * static_cast<size_t>(kRows) * BK * 2 + 2 * static_cast<size_t>(NT) * BK * 2); }

cudaError_t launch_source_angular_umma(const float* P1, const float* P2, const uint8_t* bblob, const int* groups,
                                       int n_groups, float* A1, float* A2, int* err, int nyz, int NA, int NT, int BK,
                                       int n_ntiles, cudaStream_t s) {
    if (n_groups <= 0) return cudaSuccess;
    if (BK != 32 || NT % 16 != 0 || NT < 16 || NT > 256) return cudaErrorInvalidValue;
    UmmaSourceArgs a{P1, P2, bblob, groups, A1, A2, err, nyz, NA, NT, (NA + BK - 1) / BK, n_ntiles};
    // at most two CTAs per SM when each holds 256 tensor-memory columns (512 per SM)
    size_t smem = umma_source_smem(NT, BK);
    if (NT > 128) smem = std::max<size_t>(smem, 80 * 1024);
    auto kern = source_angular_umma_kernel<32>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    dim3 grid(n_ntiles, (nyz + kPos - 1) / kPos, n_groups);
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
