// Depth-step kernels: eq15 energy sweep (with fused IDD partials), MUSCL
// predictor-corrector transport, separable DST-I angular diffusion, IDD
// finalisation, beam initialisation and conversions.
//
// State layout (HBM): index = (ek * nyz + pos) * NA + ang, ang fastest, the
// index order of the reference (bfpm_solver.cu:1996).  Every kernel walks
// ang with consecutive threads, so global accesses are coalesced.

#include "common.cuh"

#include <algorithm>
#include <cmath>

namespace bfpn {

template <typename T>
cudaError_t launch_angle_generic(const AngleArgs<T>& a, cudaStream_t s);

// ---------------------------------------------------------------------------
// Energy sweep (energyDgCnKernel, energy_solver.cu:41-161).
//
// One thread per lane (pos, ang); groups are swept from Ng-1 down to 0.  The
// recursion runs in double for both state types.  The sweep is in place: the
// old value of group ek+1 (needed by the eq15 "up" term) is kept in a
// register, the old value of group ek-1 (straggling) is the prefetched load,
// so no temporaries and no copies back are needed (the reference writes
// temporaries and copies them back, energy_solver.cu:492-505).
// Per-group constants come precomputed in a [Ng][kEnergyCoef] table; loads of
// it are uniform across the warp.
// When partials != nullptr the kernel also accumulates this species' share of
// the Eq. 24 depth dose and the psi^2 sum, and writes one pair per block.
// ---------------------------------------------------------------------------
template <int MODE, typename T>
__global__ void __launch_bounds__(256) energy_kernel(EnergyArgs<T> a) {
    const long long lane = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    double acc = 0.0, accp = 0.0;
    if (lane < a.lanes) {
        const long long L = a.lanes;
        T* __restrict__ Fp = a.F + lane;
        T* __restrict__ fp = a.f + lane;
        const T* __restrict__ sp = a.src ? a.src + lane : nullptr;
        int ek = a.Ng - 1;
        double Fn = static_cast<double>(Fp[ek * L]);
        double fn = static_cast<double>(fp[ek * L]);
        double sn = sp ? static_cast<double>(sp[ek * L]) : 0.0;
        double F_hi_old = 0.0, f_hi_old = 0.0;  // old values at ek+1
        double next_F = 0.0, next_f = 0.0;      // new values at ek+1
        double w_pos = 1.0;
        if (a.partials && a.trapezoidal) {
            const int pos = static_cast<int>(lane / a.NA);
            const int iy = pos % (a.Ny + 1), iz = pos / (a.Ny + 1);
            if (iy == 0 || iy == a.Ny) w_pos *= 0.5;
            if (iz == 0 || iz == a.Nz) w_pos *= 0.5;
        }
        for (; ek >= 0; --ek) {
            const double Fg = Fn, fg = fn, sg = sn;
            if (ek > 0) {
                Fn = static_cast<double>(Fp[(ek - 1) * L]);
                fn = static_cast<double>(fp[(ek - 1) * L]);
                if (sp) sn = static_cast<double>(sp[(ek - 1) * L]);
            }
            const double* __restrict__ c = a.coef + ek * kEnergyCoef;
            double Fv, fv;
            if (MODE == EMODE_LEGACY) {
                const double idt = __ldg(c + EC_L_IDT), hi = __ldg(c + EC_L_HI), inv = __ldg(c + EC_L_INV_DEN);
                Fv = (fmax(Fg, 0.0) * idt + hi * next_F + sg) * inv;
                fv = (fg * idt + hi * next_f) * inv;
                const double lapc = __ldg(c + EC_L_LAP);
                if (lapc > 0.0) {
                    const double Flo = (ek > 0) ? Fn : 0.0;
                    Fv += lapc * (fmax(F_hi_old, 0.0) - 2.0 * fmax(Fg, 0.0) + fmax(Flo, 0.0));
                }
                Fv = fmax(Fv, 0.0);
                fv = fmax(fv, 0.0);
            } else {
                const double up = F_hi_old - f_hi_old;
                const double cur = Fg - fg;
                double common = __ldg(c + EC_C_UP) * up + __ldg(c + EC_C_CUR) * cur + __ldg(c + EC_C_F) * Fg + sg;
                if (MODE == EMODE_EQ15_STRAG) {
                    const double Flo = (ek > 0) ? Fn : 0.0;
                    common += __ldg(c + EC_S_HI) * F_hi_old + __ldg(c + EC_S_LO) * Flo - __ldg(c + EC_S_G) * Fg;
                }
                const double hi_delta = next_F - next_f;
                const double rhs = __ldg(c + EC_R_F) * fg + __ldg(c + EC_R_UP) * up + __ldg(c + EC_R_CUR) * cur
                                 + __ldg(c + EC_R_FG) * Fg - __ldg(c + EC_A) * common + __ldg(c + EC_R_HI) * hi_delta;
                fv = rhs * __ldg(c + EC_INV_COE);
                Fv = __ldg(c + EC_F_FROM_F) * fv + __ldg(c + EC_INV_F) * common + __ldg(c + EC_F_FROM_HI) * hi_delta;
            }
            const T Fs = static_cast<T>(Fv), fs = static_cast<T>(fv);
            Fp[ek * L] = Fs;
            fp[ek * L] = fs;
            if (a.partials) {
                const double* dc = a.dose_coef + 2 * ek;
                acc += __ldg(dc) * static_cast<double>(Fs) + __ldg(dc + 1) * static_cast<double>(fs);
                accp += static_cast<double>(fs);
            }
            F_hi_old = Fg;
            f_hi_old = fg;
            next_F = Fv;
            next_f = fv;
        }
        acc *= w_pos;
    }
    if (a.partials) {
        __shared__ double red[2][32];
        for (int o = 16; o > 0; o >>= 1) {
            acc += __shfl_down_sync(0xffffffffu, acc, o);
            accp += __shfl_down_sync(0xffffffffu, accp, o);
        }
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        if (l == 0) { red[0][w] = acc; red[1][w] = accp; }
        __syncthreads();
        if (w == 0) {
            const int nw = blockDim.x >> 5;
            acc = (l < nw) ? red[0][l] : 0.0;
            accp = (l < nw) ? red[1][l] : 0.0;
            for (int o = 16; o > 0; o >>= 1) {
                acc += __shfl_down_sync(0xffffffffu, acc, o);
                accp += __shfl_down_sync(0xffffffffu, accp, o);
            }
            if (l == 0) {
                a.partials[2 * blockIdx.x] = acc;
                a.partials[2 * blockIdx.x + 1] = accp;
            }
        }
    }
}

int energy_grid(long long lanes, int block) { return static_cast<int>((lanes + block - 1) / block); }

template <typename T>
cudaError_t launch_energy(const EnergyArgs<T>& a, int block, cudaStream_t s) {
    const int grid = energy_grid(a.lanes, block);
    switch (a.mode) {
        case EMODE_EQ15: energy_kernel<EMODE_EQ15, T><<<grid, block, 0, s>>>(a); break;
        case EMODE_EQ15_STRAG: energy_kernel<EMODE_EQ15_STRAG, T><<<grid, block, 0, s>>>(a); break;
        default: energy_kernel<EMODE_LEGACY, T><<<grid, block, 0, s>>>(a); break;
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Lateral transport, Eq. (18) (spatial_transport.cu:23-161, 202-262).
//
// One block = one energy group, AC consecutive angles, one tile of output
// positions.  The block stages F over the tile plus a 4-cell halo in shared
// memory, builds the clipped predictor over the tile plus a 2-cell halo in a
// second shared buffer, and writes the corrector.  Both stencil stages and
// the two flux divergences therefore cost one HBM read and one write per
// cell (the reference does 4 launches and ~10 array passes).  Boundary
// indices clamp exactly as the reference's (max(0,i-2) .. min(Ny,i+2)).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T muscl_slope(T l, T c, T r) {
    const T fwd = r - c;
    if (fabs(fwd) < static_cast<T>(kEpsilon)) return T(0);
    const T theta = (c - l) / fwd;
    const T eta = max(T(0), max(min(T(2) * theta, T(1)), min(theta, T(2))));
    return fwd * eta;
}

template <typename T, typename Get>
__device__ __forceinline__ T flux_divergence(const Get& get, int gy, int gz, int Ny, int Nz, T wy, T wz, T dy,
                                             T dz) {
    const T c = get(gy, gz);
    const T ym2 = get(max(0, gy - 2), gz), ym1 = get(max(0, gy - 1), gz);
    const T yp1 = get(min(Ny, gy + 1), gz), yp2 = get(min(Ny, gy + 2), gz);
    T lfy, rfy;
    if (wy >= T(0)) {
        lfy = wy * (ym1 + T(0.5) * muscl_slope(ym2, ym1, c));
        rfy = wy * (c + T(0.5) * muscl_slope(ym1, c, yp1));
    } else {
        lfy = wy * (c - T(0.5) * muscl_slope(ym1, c, yp1));
        rfy = wy * (yp1 - T(0.5) * muscl_slope(c, yp1, yp2));
    }
    const T zm2 = get(gy, max(0, gz - 2)), zm1 = get(gy, max(0, gz - 1));
    const T zp1 = get(gy, min(Nz, gz + 1)), zp2 = get(gy, min(Nz, gz + 2));
    T lfz, rfz;
    if (wz >= T(0)) {
        lfz = wz * (zm1 + T(0.5) * muscl_slope(zm2, zm1, c));
        rfz = wz * (c + T(0.5) * muscl_slope(zm1, c, zp1));
    } else {
        lfz = wz * (c - T(0.5) * muscl_slope(zm1, c, zp1));
        rfz = wz * (zp1 - T(0.5) * muscl_slope(c, zp1, zp2));
    }
    return (rfy - lfy) / dy + (rfz - lfz) / dz;
}

template <typename T, int AC>
__global__ void __launch_bounds__(256) transport_kernel(TransportArgs<T> a, int tiles_y, int tiles_z, int n_chunks) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* Fs = reinterpret_cast<T*>(smem_raw);
    int b = blockIdx.x;
    const int tyi = b % tiles_y; b /= tiles_y;
    const int tzi = b % tiles_z; b /= tiles_z;
    const int chunk = b % n_chunks;
    const int ek = b / n_chunks;
    const int Ny = a.Ny, Nz = a.Nz, Ny1 = a.Ny + 1, Nz1 = a.Nz + 1, NA = a.NA;
    const int y0 = tyi * a.tile_y, y1 = min(y0 + a.tile_y, Ny1);
    const int z0 = tzi * a.tile_z, z1 = min(z0 + a.tile_z, Nz1);
    const int fy0 = max(0, y0 - 4), fy1 = min(Ny1, y1 + 4), fz0 = max(0, z0 - 4), fz1 = min(Nz1, z1 + 4);
    const int py0 = max(0, y0 - 2), py1 = min(Ny1, y1 + 2), pz0 = max(0, z0 - 2), pz1 = min(Nz1, z1 + 2);
    const int FRY = fy1 - fy0, FRZ = fz1 - fz0, PRY = py1 - py0, PRZ = pz1 - pz0;
    T* Ps = Fs + FRY * FRZ * AC;
    const int a0 = chunk * AC;
    const size_t plane = static_cast<size_t>(ek) * Ny1 * Nz1 * NA + a0;
    const T* __restrict__ in = a.in + plane;
    T* __restrict__ out = a.out + plane;

    for (int e = threadIdx.x; e < FRY * FRZ * AC; e += blockDim.x) {
        const int aa = e % AC, p = e / AC, yy = p % FRY, zz = p / FRY;
        Fs[e] = (a0 + aa < NA) ? in[(static_cast<size_t>(fz0 + zz) * Ny1 + fy0 + yy) * NA + aa] : T(0);
    }
    __syncthreads();

    const T dt = a.dt, dy = a.dy, dz = a.dz;
    for (int e = threadIdx.x; e < PRY * PRZ * AC; e += blockDim.x) {
        const int aa = e % AC, p = e / AC, yy = p % PRY, zz = p / PRY;
        const int ang = min(a0 + aa, NA - 1);
        const T wy = a.omega[2 * ang], wz = a.omega[2 * ang + 1];
        auto getF = [&](int gy, int gz) { return Fs[((gz - fz0) * FRY + (gy - fy0)) * AC + aa]; };
        const int gy = py0 + yy, gz = pz0 + zz;
        const T v = getF(gy, gz) - dt * flux_divergence<T>(getF, gy, gz, Ny, Nz, wy, wz, dy, dz);
        Ps[e] = a.preserve_sign ? v : max(v, T(0));
    }
    __syncthreads();

    const int TY = y1 - y0, TZ = z1 - z0;
    for (int e = threadIdx.x; e < TY * TZ * AC; e += blockDim.x) {
        const int aa = e % AC, p = e / AC, yy = p % TY, zz = p / TY;
        if (a0 + aa >= NA) continue;
        const int ang = a0 + aa;
        const T wy = a.omega[2 * ang], wz = a.omega[2 * ang + 1];
        auto getF = [&](int gy, int gz) { return Fs[((gz - fz0) * FRY + (gy - fy0)) * AC + aa]; };
        auto getP = [&](int gy, int gz) { return Ps[((gz - pz0) * PRY + (gy - py0)) * AC + aa]; };
        const int gy = y0 + yy, gz = z0 + zz;
        const T d0 = flux_divergence<T>(getF, gy, gz, Ny, Nz, wy, wz, dy, dz);
        const T d1 = flux_divergence<T>(getP, gy, gz, Ny, Nz, wy, wz, dy, dz);
        const T v = getF(gy, gz) - T(0.5) * dt * (d0 + d1);
        out[(static_cast<size_t>(gz) * Ny1 + gy) * NA + aa] = a.preserve_sign ? v : max(v, T(0));
    }
}

template <typename T, int AC>
static cudaError_t launch_transport_ac(const TransportArgs<T>& a, cudaStream_t s) {
    const int Ny1 = a.Ny + 1, Nz1 = a.Nz + 1;
    const int tiles_y = (Ny1 + a.tile_y - 1) / a.tile_y, tiles_z = (Nz1 + a.tile_z - 1) / a.tile_z;
    const int n_chunks = (a.NA + AC - 1) / AC;
    const int fy = std::min(Ny1, a.tile_y + 8), fz = std::min(Nz1, a.tile_z + 8);
    const int py = std::min(Ny1, a.tile_y + 4), pz = std::min(Nz1, a.tile_z + 4);
    const size_t smem = static_cast<size_t>(fy * fz + py * pz) * AC * sizeof(T);
    auto kern = transport_kernel<T, AC>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const long long blocks = static_cast<long long>(a.Ng) * n_chunks * tiles_y * tiles_z;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    kern<<<static_cast<unsigned>(blocks), 256, smem, s>>>(a, tiles_y, tiles_z, n_chunks);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_transport(const TransportArgs<T>& a, int ang_chunk, cudaStream_t s) {
    switch (ang_chunk) {
        case 4: return launch_transport_ac<T, 4>(a, s);
        case 8: return launch_transport_ac<T, 8>(a, s);
        case 16: return launch_transport_ac<T, 16>(a, s);
        case 32: return launch_transport_ac<T, 32>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------------------
// Angular diffusion, Eq. (19)-(21) (angle_diffusion.cu:7-34, 254-362).
//
// Each (ek, pos) slice X[v][u] is NA contiguous values.  One block stages
// slices_per_block slices in shared memory and applies the four separable
// DST-I passes (forward u, forward v with the CN factor, inverse v, inverse u)
// there, so the array is read once and written once (the reference makes 4
// launches through two full-size temporaries).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) angle_kernel(AngleArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int Nom = a.Nom, Nmu = a.Nmu, NA = Nom * Nmu, SL = a.slices_per_block;
    T* Su = reinterpret_cast<T*>(smem_raw);
    T* Sv = Su + Nom * Nom;
    T* X = Sv + Nmu * Nmu;
    T* Y = X + SL * NA;
    const long long total = static_cast<long long>(a.Ng) * a.nyz;
    const long long s0 = static_cast<long long>(blockIdx.x) * SL;
    const int ns = static_cast<int>(min(static_cast<long long>(SL), total - s0));
    const int n = ns * NA;
    for (int e = threadIdx.x; e < Nom * Nom; e += blockDim.x) Su[e] = a.sine_u[e];
    for (int e = threadIdx.x; e < Nmu * Nmu; e += blockDim.x) Sv[e] = a.sine_v[e];
    T* __restrict__ F = a.F + s0 * NA;
    for (int e = threadIdx.x; e < n; e += blockDim.x) X[e] = F[e];
    __syncthreads();
    for (int e = threadIdx.x; e < n; e += blockDim.x) {  // forward u
        const int s = e / NA, r = e - s * NA, v = r / Nom, mu = r - v * Nom;
        const T* x = X + s * NA + v * Nom;
        const T* su = Su + mu * Nom;
        T acc = T(0);
        for (int k = 0; k < Nom; ++k) acc += x[k] * su[k];
        Y[e] = acc;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < n; e += blockDim.x) {  // forward v, times the factor
        const int s = e / NA, r = e - s * NA, nu = r / Nom, mu = r - nu * Nom;
        const T* y = Y + s * NA + mu;
        const T* sv = Sv + nu * Nmu;
        T acc = T(0);
        for (int k = 0; k < Nmu; ++k) acc += sv[k] * y[k * Nom];
        const long long ek = (s0 + s) / a.nyz;
        X[e] = acc * a.fac[ek * NA + r];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < n; e += blockDim.x) {  // inverse v
        const int s = e / NA, r = e - s * NA, v = r / Nom, mu = r - v * Nom;
        const T* x = X + s * NA + mu;
        T acc = T(0);
        for (int k = 0; k < Nmu; ++k) acc += Sv[k * Nmu + v] * x[k * Nom];
        Y[e] = acc;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < n; e += blockDim.x) {  // inverse u
        const int s = e / NA, r = e - s * NA, v = r / Nom, u = r - v * Nom;
        const T* y = Y + s * NA + v * Nom;
        T acc = T(0);
        for (int k = 0; k < Nom; ++k) acc += y[k] * Su[k * Nom + u];
        F[e] = acc;
    }
}

// Square angular grids (Nom == Nmu == N <= 32): one thread owns a whole row
// (or column) of a slice in registers.  The DST-I matrix is symmetric and
// S[m][N-1-i] = (-1)^m S[m][i], so y = S x needs only the first ceil(N/2)
// columns applied to x[i] +- x[N-1-i]: N*ceil(N/2) FMAs per row instead of N^2.
// The half table travels by value as a kernel parameter, so its entries are
// constant-bank operands of the FMAs (no shared-memory traffic for it).
template <int N, typename T>
struct SineHalf {
    T h[N][(N + 1) / 2];
};

template <int N, typename T>
__device__ __forceinline__ void dst1(const SineHalf<N, T>& S, const T (&x)[N], T (&y)[N]) {
    constexpr int H = N / 2, HC = (N + 1) / 2;
    T p[HC], q[H > 0 ? H : 1];
#pragma unroll
    for (int i = 0; i < H; ++i) {
        p[i] = x[i] + x[N - 1 - i];
        q[i] = x[i] - x[N - 1 - i];
    }
    if (N & 1) p[H] = x[H];
#pragma unroll
    for (int m = 0; m < N; ++m) {
        T acc = T(0);
        if ((m & 1) == 0) {
#pragma unroll
            for (int i = 0; i < HC; ++i) acc += S.h[m][i] * p[i];
        } else {
#pragma unroll
            for (int i = 0; i < H; ++i) acc += S.h[m][i] * q[i];
        }
        y[m] = acc;
    }
}

template <int N, typename T>
__global__ void __launch_bounds__(256) angle_dst_kernel(AngleArgs<T> a, SineHalf<N, T> S) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NA = N * N, RS = N + 1;  // padded row stride: conflict-free row and column access
    T* X = reinterpret_cast<T*>(smem_raw);
    const int SL = a.slices_per_block;
    const long long total = static_cast<long long>(a.Ng) * a.nyz;
    const long long s0 = static_cast<long long>(blockIdx.x) * SL;
    const int ns = static_cast<int>(min(static_cast<long long>(SL), total - s0));
    T* __restrict__ F = a.F + s0 * NA;
    for (int e = threadIdx.x; e < ns * NA; e += blockDim.x) {
        const int s = e / NA, r = e - s * NA, v = r / N, u = r - v * N;
        X[(s * N + v) * RS + u] = F[e];
    }
    __syncthreads();
    T x[N], y[N];
    for (int row = threadIdx.x; row < ns * N; row += blockDim.x) {  // forward u
        T* R = X + row * RS;
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = R[k];
        dst1<N, T>(S, x, y);
#pragma unroll
        for (int k = 0; k < N; ++k) R[k] = y[k];
    }
    __syncthreads();
    for (int col = threadIdx.x; col < ns * N; col += blockDim.x) {  // forward v, factor, inverse v
        const int s = col / N, mu = col - s * N;
        T* C = X + s * N * RS + mu;
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = C[k * RS];
        dst1<N, T>(S, x, y);
        const T* __restrict__ fac = a.fac + ((s0 + s) / a.nyz) * NA + mu;
#pragma unroll
        for (int k = 0; k < N; ++k) y[k] *= fac[k * N];
        dst1<N, T>(S, y, x);
#pragma unroll
        for (int k = 0; k < N; ++k) C[k * RS] = x[k];
    }
    __syncthreads();
    for (int row = threadIdx.x; row < ns * N; row += blockDim.x) {  // inverse u
        T* R = X + row * RS;
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = R[k];
        dst1<N, T>(S, x, y);
#pragma unroll
        for (int k = 0; k < N; ++k) R[k] = y[k];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < ns * NA; e += blockDim.x) {
        const int s = e / NA, r = e - s * NA, v = r / N, u = r - v * N;
        F[e] = X[(s * N + v) * RS + u];
    }
}

template <int N, typename T>
static cudaError_t launch_angle_dst(const AngleArgs<T>& a, cudaStream_t s) {
    SineHalf<N, T> S;
    // sine_u lives on the device; the host copy of the half table is built
    // from the same formula the tables use (angle_diffusion.cu:393-397).
    for (int m = 0; m < N; ++m)
        for (int i = 0; i < (N + 1) / 2; ++i)
            S.h[m][i] = static_cast<T>(std::sin(3.14159265358979323846 * (m + 1) * (i + 1) / (N + 1)));
    const int SL = std::max(1, 256 / N);
    const size_t smem = static_cast<size_t>(SL) * N * (N + 1) * sizeof(T);
    auto kern = angle_dst_kernel<N, T>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    AngleArgs<T> b = a;
    b.slices_per_block = SL;
    const long long total = static_cast<long long>(a.Ng) * a.nyz;
    const long long blocks = (total + SL - 1) / SL;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    kern<<<static_cast<unsigned>(blocks), 256, smem, s>>>(b, S);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_angle(const AngleArgs<T>& a, cudaStream_t s) {
    if (a.Nom == a.Nmu) {
        switch (a.Nom) {
#define BFPN_DST_CASE(n) \
    case n: return launch_angle_dst<n, T>(a, s);
            BFPN_DST_CASE(2) BFPN_DST_CASE(3) BFPN_DST_CASE(4) BFPN_DST_CASE(5) BFPN_DST_CASE(6) BFPN_DST_CASE(7)
            BFPN_DST_CASE(8) BFPN_DST_CASE(9) BFPN_DST_CASE(10) BFPN_DST_CASE(11) BFPN_DST_CASE(12)
            BFPN_DST_CASE(13) BFPN_DST_CASE(14) BFPN_DST_CASE(15) BFPN_DST_CASE(16) BFPN_DST_CASE(17)
            BFPN_DST_CASE(18) BFPN_DST_CASE(19) BFPN_DST_CASE(20) BFPN_DST_CASE(21) BFPN_DST_CASE(22)
            BFPN_DST_CASE(23) BFPN_DST_CASE(24) BFPN_DST_CASE(28) BFPN_DST_CASE(32)
#undef BFPN_DST_CASE
            default: break;
        }
    }
    return launch_angle_generic(a, s);
}

template <typename T>
cudaError_t launch_angle_generic(const AngleArgs<T>& a, cudaStream_t s) {
    const int NA = a.Nom * a.Nmu;
    const size_t smem = (static_cast<size_t>(a.Nom) * a.Nom + static_cast<size_t>(a.Nmu) * a.Nmu
                         + 2 * static_cast<size_t>(a.slices_per_block) * NA) * sizeof(T);
    auto kern = angle_kernel<T>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const long long total = static_cast<long long>(a.Ng) * a.nyz;
    const long long blocks = (total + a.slices_per_block - 1) / a.slices_per_block;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    kern<<<static_cast<unsigned>(blocks), 256, smem, s>>>(a);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// IDD: stand-alone partials (for a species whose last energy pass did not
// fuse them) and the deterministic final sum into the device history.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) idd_partials_kernel(const T* __restrict__ F, const T* __restrict__ f,
                                                           const double* __restrict__ dc, int Ng, long long lanes,
                                                           int NA, int Ny, int Nz, int trap, int with_proxy,
                                                           double* partials) {
    double acc = 0.0, accp = 0.0;
    for (long long lane = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; lane < lanes;
         lane += static_cast<long long>(gridDim.x) * blockDim.x) {
        double w = 1.0;
        if (trap) {
            const int pos = static_cast<int>(lane / NA), iy = pos % (Ny + 1), iz = pos / (Ny + 1);
            if (iy == 0 || iy == Ny) w *= 0.5;
            if (iz == 0 || iz == Nz) w *= 0.5;
        }
        double part = 0.0;
        for (int ek = 0; ek < Ng; ++ek) {
            const double x = static_cast<double>(F[ek * lanes + lane]);
            const double y = static_cast<double>(f[ek * lanes + lane]);
            part += dc[2 * ek] * x + dc[2 * ek + 1] * y;
            accp += y;
        }
        acc += w * part;
    }
    if (!with_proxy) accp = 0.0;
    __shared__ double red[2][32];
    for (int o = 16; o > 0; o >>= 1) {
        acc += __shfl_down_sync(0xffffffffu, acc, o);
        accp += __shfl_down_sync(0xffffffffu, accp, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { red[0][w] = acc; red[1][w] = accp; }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        acc = (l < nw) ? red[0][l] : 0.0;
        accp = (l < nw) ? red[1][l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            acc += __shfl_down_sync(0xffffffffu, acc, o);
            accp += __shfl_down_sync(0xffffffffu, accp, o);
        }
        if (l == 0) { partials[2 * blockIdx.x] = acc; partials[2 * blockIdx.x + 1] = accp; }
    }
}

int idd_partials_grid(long long lanes) {
    long long g = (lanes + 255) / 256;
    return static_cast<int>(std::min<long long>(std::max<long long>(g, 1), 4 * 148));
}

template <typename T>
cudaError_t launch_idd_partials(const T* F, const T* f, const double* dc, int Ng, long long lanes, int NA, int Ny,
                                int Nz, int trap, int with_proxy, double* partials, int grid, cudaStream_t s) {
    idd_partials_kernel<T><<<grid, 256, 0, s>>>(F, f, dc, Ng, lanes, NA, Ny, Nz, trap, with_proxy, partials);
    return cudaGetLastError();
}

__global__ void __launch_bounds__(1024) finalize_idd_kernel(const double* __restrict__ p, int n,
                                                            const double* __restrict__ p2, int n2,
                                                            double idd_scale, double proxy_scale,
                                                            double* hist_idd, double* hist_proxy, int* counter,
                                                            int capacity, int advance) {
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) { a += p[2 * i]; b += p[2 * i + 1]; }
    for (int i = threadIdx.x; i < n2; i += blockDim.x) a += p2[2 * i];  // psi^2 sum: primary only
    __shared__ double red[2][32];
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { red[0][w] = a; red[1][w] = b; }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        a = (l < nw) ? red[0][l] : 0.0;
        b = (l < nw) ? red[1][l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if (l == 0) {
            const int c = *counter;
            if (c >= 0 && c < capacity) {
                hist_idd[c] = a * idd_scale;
                hist_proxy[c] = b * proxy_scale;
            }
            if (advance) *counter = c + 1;
        }
    }
}

cudaError_t launch_finalize_idd(const double* partials, int n, const double* partials2, int n2, double idd_scale,
                                double proxy_scale, double* hist_idd, double* hist_proxy, int* counter,
                                int capacity, int advance, cudaStream_t s) {
    finalize_idd_kernel<<<1, 1024, 0, s>>>(partials, n, partials2, n2, idd_scale, proxy_scale, hist_idd, hist_proxy,
                                           counter, capacity, advance);
    return cudaGetLastError();
}

// energyMomentKernel (bfpm_solver.cu:311-360): one block per group.
template <typename T>
__global__ void __launch_bounds__(256) energy_moments_kernel(const T* F, const T* f, const T* F1, const T* f1,
                                                             long long per_e, double weight, double* out) {
    const int ek = blockIdx.x;
    double s1 = 0.0, s2 = 0.0;
    const long long base = static_cast<long long>(ek) * per_e;
    for (long long l = threadIdx.x; l < per_e; l += blockDim.x) {
        s1 += static_cast<double>(F[base + l]) + static_cast<double>(F1[base + l]);
        s2 += static_cast<double>(f[base + l]) + static_cast<double>(f1[base + l]);
    }
    __shared__ double red[2][32];
    for (int o = 16; o > 0; o >>= 1) {
        s1 += __shfl_down_sync(0xffffffffu, s1, o);
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { red[0][w] = s1; red[1][w] = s2; }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        s1 = (l < nw) ? red[0][l] : 0.0;
        s2 = (l < nw) ? red[1][l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            s1 += __shfl_down_sync(0xffffffffu, s1, o);
            s2 += __shfl_down_sync(0xffffffffu, s2, o);
        }
        if (l == 0) { out[2 * ek] = s1 * weight; out[2 * ek + 1] = s2 * weight; }
    }
}

template <typename T>
cudaError_t launch_energy_moments(const T* F, const T* f, const T* F1, const T* f1, int Ng, long long per_e,
                                  double weight, double* out, cudaStream_t s) {
    energy_moments_kernel<T><<<Ng, 256, 0, s>>>(F, f, F1, f1, per_e, weight, out);
    return cudaGetLastError();
}

// Initial beam, full mode (bfpm_solver.cu:1966-2000): F = f1(pos, ang) * f2(ek),
// the product of the two factors evaluated on the host exactly as there.
template <typename T>
__global__ void init_beam_kernel(T* F, const double* __restrict__ yza, const double* __restrict__ e, long long per_e,
                                 long long total) {
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long ek = i / per_e, l = i - ek * per_e;
        F[i] = static_cast<T>(yza[l] * e[ek]);
    }
}

template <typename T>
cudaError_t launch_init_beam(T* F, const double* yza, const double* e, long long per_e, int Ng, cudaStream_t s) {
    const long long total = per_e * Ng;
    const int grid = static_cast<int>(std::min<long long>((total + 255) / 256, 148 * 16));
    init_beam_kernel<T><<<grid, 256, 0, s>>>(F, yza, e, per_e, total);
    return cudaGetLastError();
}

template <typename Tin, typename Tout>
__global__ void convert_kernel(const Tin* in, Tout* out, long long n) {
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        out[i] = static_cast<Tout>(in[i]);
}

template <typename Tin, typename Tout>
cudaError_t launch_convert(const Tin* in, Tout* out, long long n, cudaStream_t s) {
    const int grid = static_cast<int>(std::min<long long>(std::max<long long>((n + 255) / 256, 1), 148 * 16));
    convert_kernel<Tin, Tout><<<grid, 256, 0, s>>>(in, out, n);
    return cudaGetLastError();
}

#define BFPN_INSTANTIATE(T)                                                                                       \
    template cudaError_t launch_energy<T>(const EnergyArgs<T>&, int, cudaStream_t);                               \
    template cudaError_t launch_transport<T>(const TransportArgs<T>&, int, cudaStream_t);                         \
    template cudaError_t launch_angle<T>(const AngleArgs<T>&, cudaStream_t);                                      \
    template cudaError_t launch_idd_partials<T>(const T*, const T*, const double*, int, long long, int, int, int,  \
                                                int, int, double*, int, cudaStream_t);                            \
    template cudaError_t launch_energy_moments<T>(const T*, const T*, const T*, const T*, int, long long, double, \
                                                  double*, cudaStream_t);                                         \
    template cudaError_t launch_init_beam<T>(T*, const double*, const double*, long long, int, cudaStream_t);

BFPN_INSTANTIATE(double)
BFPN_INSTANTIATE(float)
template cudaError_t launch_convert<double, float>(const double*, float*, long long, cudaStream_t);
template cudaError_t launch_convert<float, double>(const float*, double*, long long, cudaStream_t);
template cudaError_t launch_convert<double, double>(const double*, double*, long long, cudaStream_t);

}  // namespace bfpn
