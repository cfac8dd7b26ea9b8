// Catastrophic secondary source (secondarySourceFromPrimaryKernel,
// energy_solver.cu:287-333):
//
//   S[e, pos, out] = dg * sum_{s in band(e)} sum_in ker_v[s, in, out]
//                      * (e1[e, s] * max(P1[s, pos, in], 0) + e2[e, s] * P2[s, pos, in] / 3)
//
// factorised into two contractions that each read their operands once:
//   A1[s, pos, out] = sum_in max(P1[s, pos, in], 0) * ker_v[s, in, out]   (angular GEMM per source group)
//   A2[s, pos, out] = sum_in P2[s, pos, in] * ker_v[s, in, out]
//   S[e, l]         = dg * (sum_s e1[e, s] A1[s, l] + (sum_s e2[e, s] A2[s, l]) / 3)   (banded energy GEMM)
// The reference re-reads the primary band*NA times per output cell.

#include "common.cuh"

#include <algorithm>

namespace bfpn {

// Angular stage: per source group g, C[pos][out] = X[pos][in] * K[in][out]
// for X = max(P1, 0) and X = P2 at once (they share the K tiles).
// 64 x 64 output tile per block, 16 x 16 threads, 4 x 4 outputs per thread
// per operand, K staged through shared memory 16 deep.
template <typename T>
__global__ void __launch_bounds__(256) source_angular_kernel(SourceArgs<T> a) {
    constexpr int BM = 64, BN = 64, BK = 16;
    __shared__ T X1s[BK][BM + 1];
    __shared__ T X2s[BK][BM + 1];
    __shared__ T Ks[BK][BN];
    const int g = a.groups[blockIdx.z];
    const int NA = a.NA, nyz = a.nyz;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const T* __restrict__ P1 = a.P1 + static_cast<size_t>(g) * nyz * NA;
    const T* __restrict__ P2 = a.P2 + static_cast<size_t>(g) * nyz * NA;
    const T* __restrict__ K = a.ker_v + static_cast<size_t>(g) * NA * NA;
    T acc1[4][4], acc2[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) { acc1[i][j] = T(0); acc2[i][j] = T(0); }

    for (int k0 = 0; k0 < NA; k0 += BK) {
        for (int e = threadIdx.x; e < BM * BK; e += 256) {
            const int k = e % BK, m = e / BK;
            const int gm = m0 + m, gk = k0 + k;
            T x1 = T(0), x2 = T(0);
            if (gm < nyz && gk < NA) {
                x1 = P1[static_cast<size_t>(gm) * NA + gk];
                x2 = P2[static_cast<size_t>(gm) * NA + gk];
            }
            X1s[k][m] = max(x1, T(0));
            X2s[k][m] = x2;
        }
        for (int e = threadIdx.x; e < BK * BN; e += 256) {
            const int n = e % BN, k = e / BN;
            const int gn = n0 + n, gk = k0 + k;
            Ks[k][n] = (gn < NA && gk < NA) ? K[static_cast<size_t>(gk) * NA + gn] : T(0);
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < BK; ++k) {
            T x1[4], x2[4], kv[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) { x1[i] = X1s[k][ty + 16 * i]; x2[i] = X2s[k][ty + 16 * i]; }
#pragma unroll
            for (int j = 0; j < 4; ++j) kv[j] = Ks[k][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    acc1[i][j] += x1[i] * kv[j];
                    acc2[i][j] += x2[i] * kv[j];
                }
        }
        __syncthreads();
    }
    T* __restrict__ A1 = a.A1 + static_cast<size_t>(g) * nyz * NA;
    T* __restrict__ A2 = a.A2 + static_cast<size_t>(g) * nyz * NA;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gm = m0 + ty + 16 * i;
        if (gm >= nyz) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int gn = n0 + tx + 16 * j;
            if (gn < NA) {
                A1[static_cast<size_t>(gm) * NA + gn] = acc1[i][j];
                A2[static_cast<size_t>(gm) * NA + gn] = acc2[i][j];
            }
        }
    }
}

template <typename T>
cudaError_t launch_source_angular(const SourceArgs<T>& a, cudaStream_t s) {
    if (a.n_groups <= 0) return cudaSuccess;
    dim3 grid((a.NA + 63) / 64, (a.nyz + 63) / 64, a.n_groups);
    source_angular_kernel<T><<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

// Float state: the same contraction on packed fp32x2 FMAs.  Accumulators
// pair neighbouring output groups of one lane, so one instruction applies the
// coefficients of outputs (2t, 2t+1) -- one 8-byte piece of a shared-memory
// row -- to the lane's value held twice.  Products and sums are the scalar
// kernel's, output by output.
template <int TE, int LN>
__global__ void __launch_bounds__(128) source_energy_f2_kernel(SourceArgs<float> a) {
    constexpr int SC = 32, TP = TE / 2;
    __shared__ __align__(16) float E1[SC][TE];
    __shared__ __align__(16) float E2[SC][TE];
    const int tile = blockIdx.x;
    const long long per_e = static_cast<long long>(a.nyz) * a.NA;
    const long long l0 = static_cast<long long>(blockIdx.y) * blockDim.x * LN + threadIdx.x;
    const int Ng = a.Ng, e0 = tile * TE;
    const int lo = a.tile_lo[tile], hi = a.tile_hi[tile];
    float2 q1[TP][LN], q2[TP][LN];
#pragma unroll
    for (int t = 0; t < TP; ++t)
#pragma unroll
        for (int j = 0; j < LN; ++j) q1[t][j] = q2[t][j] = make_float2(0.f, 0.f);
    long long lj[LN];
    bool ok[LN];
#pragma unroll
    for (int j = 0; j < LN; ++j) {
        lj[j] = l0 + static_cast<long long>(j) * blockDim.x;
        ok[j] = lj[j] < per_e;
    }
    for (int s0 = lo; s0 < hi; s0 += SC) {
        const int n = min(SC, hi - s0);
        __syncthreads();
        for (int k = threadIdx.x; k < SC * TE; k += blockDim.x) {
            const int ss = k / TE, t = k - ss * TE, e = e0 + t;
            const bool in = ss < n && e < Ng;
            E1[ss][t] = in ? static_cast<float>(a.e1[static_cast<size_t>(e) * Ng + s0 + ss]) : 0.f;
            E2[ss][t] = in ? static_cast<float>(a.e2[static_cast<size_t>(e) * Ng + s0 + ss]) : 0.f;
        }
        __syncthreads();
#pragma unroll 2
        for (int ss = 0; ss < n; ++ss) {
            const long long row = static_cast<long long>(s0 + ss) * per_e;
            float2 x1[LN], x2[LN];
#pragma unroll
            for (int j = 0; j < LN; ++j) {
                const float v1 = ok[j] ? a.A1[row + lj[j]] : 0.f, v2 = ok[j] ? a.A2[row + lj[j]] : 0.f;
                x1[j] = make_float2(v1, v1);
                x2[j] = make_float2(v2, v2);
            }
            const float2* c1 = reinterpret_cast<const float2*>(E1[ss]);
            const float2* c2 = reinterpret_cast<const float2*>(E2[ss]);
#pragma unroll
            for (int t = 0; t < TP; ++t) {
                const float2 a1 = c1[t], a2 = c2[t];
#pragma unroll
                for (int j = 0; j < LN; ++j) {
                    q1[t][j] = __ffma2_rn(a1, x1[j], q1[t][j]);
                    q2[t][j] = __ffma2_rn(a2, x2[j], q2[t][j]);
                }
            }
        }
    }
    const float dg = static_cast<float>(a.dg), third = 1.f / 3.f;
#pragma unroll
    for (int t = 0; t < TP; ++t)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int e = e0 + 2 * t + h;
            if (e >= Ng) continue;
#pragma unroll
            for (int j = 0; j < LN; ++j)
                if (ok[j]) {
                    const float s1 = h ? q1[t][j].y : q1[t][j].x, s2 = h ? q2[t][j].y : q2[t][j].x;
                    a.S[e * per_e + lj[j]] = dg * (s1 + s2 * third);
                }
        }
}

// Energy stage: TE output groups per block and LN lanes per thread.  The
// source groups of the union band of the TE outputs are streamed once; the
// band coefficients of a chunk of SC source groups are staged in shared
// memory as [s][t] rows (one vector broadcast load feeds 4 (float) or 2
// (double) accumulators), and zeros outside an output's own band add
// nothing.  Accumulation in the state precision; blockIdx.x walks the output
// tiles so blocks sharing a lane range run together and share A rows in L2.
template <typename T, int TE, int LN>
__global__ void __launch_bounds__(128) source_energy_kernel(SourceArgs<T> a) {
    constexpr int SC = 32;
    __shared__ __align__(16) T E1[SC][TE];
    __shared__ __align__(16) T E2[SC][TE];
    const int tile = blockIdx.x;
    const long long per_e = static_cast<long long>(a.nyz) * a.NA;
    const long long l0 = static_cast<long long>(blockIdx.y) * blockDim.x * LN + threadIdx.x;
    const int Ng = a.Ng, e0 = tile * TE;
    const int lo = a.tile_lo[tile], hi = a.tile_hi[tile];
    T q1[TE][LN], q2[TE][LN];
#pragma unroll
    for (int t = 0; t < TE; ++t)
#pragma unroll
        for (int j = 0; j < LN; ++j) { q1[t][j] = T(0); q2[t][j] = T(0); }
    long long lj[LN];
    bool ok[LN];
#pragma unroll
    for (int j = 0; j < LN; ++j) {
        lj[j] = l0 + static_cast<long long>(j) * blockDim.x;
        ok[j] = lj[j] < per_e;
    }
    for (int s0 = lo; s0 < hi; s0 += SC) {
        const int n = min(SC, hi - s0);
        __syncthreads();
        for (int k = threadIdx.x; k < SC * TE; k += blockDim.x) {
            const int ss = k / TE, t = k - ss * TE, e = e0 + t;
            const bool in = ss < n && e < Ng;
            E1[ss][t] = in ? static_cast<T>(a.e1[static_cast<size_t>(e) * Ng + s0 + ss]) : T(0);
            E2[ss][t] = in ? static_cast<T>(a.e2[static_cast<size_t>(e) * Ng + s0 + ss]) : T(0);
        }
        __syncthreads();
#pragma unroll 2
        for (int ss = 0; ss < n; ++ss) {
            T x1[LN], x2[LN];
            const long long row = static_cast<long long>(s0 + ss) * per_e;
#pragma unroll
            for (int j = 0; j < LN; ++j) {
                x1[j] = ok[j] ? a.A1[row + lj[j]] : T(0);
                x2[j] = ok[j] ? a.A2[row + lj[j]] : T(0);
            }
#pragma unroll
            for (int t = 0; t < TE; ++t) {
                const T c1 = E1[ss][t], c2 = E2[ss][t];
#pragma unroll
                for (int j = 0; j < LN; ++j) {
                    q1[t][j] += c1 * x1[j];
                    q2[t][j] += c2 * x2[j];
                }
            }
        }
    }
    const T dg = static_cast<T>(a.dg), third = T(1) / T(3);
#pragma unroll
    for (int t = 0; t < TE; ++t) {
        const int e = e0 + t;
        if (e >= Ng) continue;
#pragma unroll
        for (int j = 0; j < LN; ++j)
            if (ok[j]) a.S[e * per_e + lj[j]] = dg * (q1[t][j] + q2[t][j] * third);
    }
}

template <typename T>
cudaError_t launch_source_energy(const SourceArgs<T>& a, int tile_e, cudaStream_t s) {
    constexpr int LN = sizeof(T) == 4 ? 2 : 1;
    const long long per_e = static_cast<long long>(a.nyz) * a.NA;
    const int tiles = (a.Ng + tile_e - 1) / tile_e;
    const long long ly = (per_e + 128 * LN - 1) / (128 * LN);
    if (ly > 65535) return cudaErrorInvalidConfiguration;
    dim3 grid(tiles, static_cast<unsigned>(ly));
    if constexpr (sizeof(T) == 4) {
        switch (tile_e) {
            case 8: source_energy_f2_kernel<8, LN><<<grid, 128, 0, s>>>(a); break;
            case 16: source_energy_f2_kernel<16, LN><<<grid, 128, 0, s>>>(a); break;
            default: return cudaErrorInvalidValue;
        }
    } else {
        switch (tile_e) {
            case 8: source_energy_kernel<T, 8, LN><<<grid, 128, 0, s>>>(a); break;
            case 16: source_energy_kernel<T, 16, LN><<<grid, 128, 0, s>>>(a); break;
            default: return cudaErrorInvalidValue;
        }
    }
    return cudaGetLastError();
}

template cudaError_t launch_source_angular<double>(const SourceArgs<double>&, cudaStream_t);
template cudaError_t launch_source_angular<float>(const SourceArgs<float>&, cudaStream_t);
template cudaError_t launch_source_energy<double>(const SourceArgs<double>&, int, cudaStream_t);
template cudaError_t launch_source_energy<float>(const SourceArgs<float>&, int, cudaStream_t);

}  // namespace bfpn
