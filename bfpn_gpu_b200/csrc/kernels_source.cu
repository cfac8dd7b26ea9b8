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

// Energy stage: one thread per lane, TE output groups per block; the source
// groups of the union band of those outputs are streamed once and applied to
// all TE accumulators (zeros outside each output's band contribute nothing).
// Accumulation in double; blockIdx.x walks the output tiles so that blocks
// sharing a lane range run together and share A rows through L2.
template <typename T, int TE>
__global__ void __launch_bounds__(128) source_energy_kernel(SourceArgs<T> a) {
    const int tile = blockIdx.x;
    const long long per_e = static_cast<long long>(a.nyz) * a.NA;
    const long long l = static_cast<long long>(blockIdx.y) * blockDim.x + threadIdx.x;
    if (l >= per_e) return;
    const int Ng = a.Ng, e0 = tile * TE;
    const int lo = a.tile_lo[tile], hi = a.tile_hi[tile];
    double q1[TE], q2[TE];
#pragma unroll
    for (int t = 0; t < TE; ++t) { q1[t] = 0.0; q2[t] = 0.0; }
    for (int s = lo; s < hi; ++s) {
        const double x1 = static_cast<double>(a.A1[s * per_e + l]);
        const double x2 = static_cast<double>(a.A2[s * per_e + l]);
#pragma unroll
        for (int t = 0; t < TE; ++t) {
            const int e = min(e0 + t, Ng - 1);
            q1[t] += __ldg(a.e1 + static_cast<size_t>(e) * Ng + s) * x1;
            q2[t] += __ldg(a.e2 + static_cast<size_t>(e) * Ng + s) * x2;
        }
    }
#pragma unroll
    for (int t = 0; t < TE; ++t) {
        const int e = e0 + t;
        if (e < Ng) a.S[e * per_e + l] = static_cast<T>(a.dg * (q1[t] + q2[t] / 3.0));
    }
}

template <typename T>
cudaError_t launch_source_energy(const SourceArgs<T>& a, int tile_e, cudaStream_t s) {
    const long long per_e = static_cast<long long>(a.nyz) * a.NA;
    const int tiles = (a.Ng + tile_e - 1) / tile_e;
    dim3 grid(tiles, static_cast<unsigned>((per_e + 127) / 128));
    switch (tile_e) {
        case 8: source_energy_kernel<T, 8><<<grid, 128, 0, s>>>(a); break;
        case 16: source_energy_kernel<T, 16><<<grid, 128, 0, s>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template cudaError_t launch_source_angular<double>(const SourceArgs<double>&, cudaStream_t);
template cudaError_t launch_source_angular<float>(const SourceArgs<float>&, cudaStream_t);
template cudaError_t launch_source_energy<double>(const SourceArgs<double>&, int, cudaStream_t);
template cudaError_t launch_source_energy<float>(const SourceArgs<float>&, int, cudaStream_t);

}  // namespace bfpn
