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
#include <cstring>

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
        const int Ng = a.Ng;
        // ring of the next D groups' old values, loaded D groups ahead of use
        constexpr int D = 8;
        T rF[D], rf[D], rs[D];
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const int e = Ng - 1 - k;
            rF[k] = e >= 0 ? Fp[e * L] : T(0);
            rf[k] = e >= 0 ? fp[e * L] : T(0);
            rs[k] = (e >= 0 && sp) ? sp[e * L] : T(0);
        }
        double F_hi_old = 0.0, f_hi_old = 0.0;  // old values at ek+1
        double next_F = 0.0, next_f = 0.0;      // new values at ek+1
        double w_pos = 1.0;
        if (a.partials && a.trapezoidal) {
            const int pos = static_cast<int>(lane / a.NA);
            const int iy = pos % (a.Ny + 1), iz = pos / (a.Ny + 1);
            if (iy == 0 || iy == a.Ny) w_pos *= 0.5;
            if (iz == 0 || iz == a.Nz) w_pos *= 0.5;
        }
        for (int base = Ng - 1; base >= 0; base -= D)
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const int ek = base - k;
            if (ek < 0) break;
            const double Fg = static_cast<double>(rF[k]), fg = static_cast<double>(rf[k]),
                         sg = static_cast<double>(rs[k]);
            const int ep = ek - D;  // refill this slot D groups ahead
            if (ep >= 0) {
                rF[k] = Fp[ep * L];
                rf[k] = fp[ep * L];
                if (sp) rs[k] = sp[ep * L];
            }
            // old value of group ek-1 (straggling): the next slot, or the refill of slot 0
            const double Fn = static_cast<double>(rF[(k + 1) % D]);
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
// MUSCL slope of the reference (muscl_paper_slope, spatial_transport.cu:23-29):
// fwd * max(0, max(min(2 theta, 1), min(theta, 2))) with theta = back / fwd,
// and 0 when |fwd| < 1e-10.  Written without the division: with
// sg = sign(fwd) and b = sg * back, the limited slope is
// sg * max(0, max(min(2b, |fwd|), min(b, 2|fwd|))) -- case by case equal to
// fwd * eta (theta <= 0, <= 1/2, <= 1, <= 2, > 2).
template <typename T>
__device__ __forceinline__ T superbee(T l, T c, T r) {
    const T fwd = r - c;
    const T sg = fwd >= T(0) ? T(1) : T(-1);
    const T af = fabs(fwd), b = sg * (c - l);
    const T m = max(T(0), max(min(T(2) * b, af), min(b, T(2) * af)));
    return af < static_cast<T>(kEpsilon) ? T(0) : sg * m;
}

// A rectangle of positions [y0, y1) x [z0, z1) staged in shared memory with
// AC angles per position (angle fastest).
struct Rect {
    int y0, y1, z0, z1;
    __device__ int w() const { return y1 - y0; }
    __device__ int n() const { return (y1 - y0) * (z1 - z0); }
    __device__ int at(int gy, int gz) const { return (gz - z0) * (y1 - y0) + (gy - y0); }
    __device__ Rect grow(int h, int Ny1, int Nz1) const {
        return Rect{max(0, y0 - h), min(Ny1, y1 + h), max(0, z0 - h), min(Nz1, z1 + h)};
    }
};

// position index p of a rectangle -> global (gy, gz); w < 2^12 so the float
// quotient is exact after truncation
__device__ __forceinline__ void rect_pos(const Rect& r, int p, float inv_w, int& gy, int& gz) {
    const int zz = __float2int_rz((p + 0.5f) * inv_w);
    gz = r.z0 + zz;
    gy = r.y0 + p - zz * r.w();
}

// AC consecutive values of one position in shared memory (16-byte aligned).
template <typename T, int AC>
struct Vec {
    T v[AC];
};
template <typename T, int AC>
__device__ __forceinline__ void lds(const T* p, T (&v)[AC]) {
    if (sizeof(T) * AC % 16 == 0) {
#pragma unroll
        for (int q = 0; q < AC; q += 16 / sizeof(T)) {
            const float4 x = *reinterpret_cast<const float4*>(p + q);
            memcpy(&v[q], &x, 16);
        }
    } else {
#pragma unroll
        for (int q = 0; q < AC; ++q) v[q] = p[q];
    }
}
template <typename T, int AC>
__device__ __forceinline__ void sts(T* p, const T (&v)[AC]) {
    if (sizeof(T) * AC % 16 == 0) {
#pragma unroll
        for (int q = 0; q < AC; q += 16 / sizeof(T)) {
            float4 x;
            memcpy(&x, &v[q], 16);
            *reinterpret_cast<float4*>(p + q) = x;
        }
    } else {
#pragma unroll
        for (int q = 0; q < AC; ++q) p[q] = v[q];
    }
}

// Face values of X over `region` (X staged over rx, which holds every clamped
// neighbour): Gy = X + 0.5 sgn(wy) s_y, Gz likewise; one thread per position,
// all AC angles of it.
template <typename T, int AC>
__device__ __forceinline__ void build_faces(const T* X, const Rect& rx, T* Gy, T* Gz, const Rect& rg,
                                            const Rect& region, int Ny, int Nz, const T (&hy)[AC], const T (&hz)[AC]) {
    const float inv_w = 1.0f / region.w();
    for (int p = threadIdx.x; p < region.n(); p += blockDim.x) {
        int gy, gz;
        rect_pos(region, p, inv_w, gy, gz);
        T c[AC], m[AC], n[AC], fy[AC], fz[AC];
        lds<T, AC>(X + rx.at(gy, gz) * AC, c);
        lds<T, AC>(X + rx.at(max(0, gy - 1), gz) * AC, m);
        lds<T, AC>(X + rx.at(min(Ny, gy + 1), gz) * AC, n);
#pragma unroll
        for (int q = 0; q < AC; ++q) fy[q] = c[q] + hy[q] * superbee(m[q], c[q], n[q]);
        lds<T, AC>(X + rx.at(gy, max(0, gz - 1)) * AC, m);
        lds<T, AC>(X + rx.at(gy, min(Nz, gz + 1)) * AC, n);
#pragma unroll
        for (int q = 0; q < AC; ++q) fz[q] = c[q] + hz[q] * superbee(m[q], c[q], n[q]);
        sts<T, AC>(Gy + rg.at(gy, gz) * AC, fy);
        sts<T, AC>(Gz + rg.at(gy, gz) * AC, fz);
    }
}

// Upwind flux divergence of X at (gy, gz), all AC angles, from the face
// values G = X + 0.5 sgn(omega) slope (spatial_flux_divergence_value,
// spatial_transport.cu:31-102).  At a boundary the reference's clamped
// stencil makes the outer face value X itself (the slope of a constant
// triple is 0).
template <typename T, int AC>
__device__ __forceinline__ void face_divergence(const T* X, const Rect& rx, const T* Gy, const T* Gz, const Rect& rg,
                                                int gy, int gz, int Ny, int Nz, const T (&wy)[AC], const T (&wz)[AC],
                                                T rdy, T rdz, T (&div)[AC]) {
    T c[AC], l[AC], r[AC];
    lds<T, AC>(Gy + rg.at(gy, gz) * AC, c);
    lds<T, AC>(gy > 0 ? Gy + rg.at(gy - 1, gz) * AC : X + rx.at(0, gz) * AC, l);
    lds<T, AC>(gy < Ny ? Gy + rg.at(gy + 1, gz) * AC : X + rx.at(Ny, gz) * AC, r);
#pragma unroll
    for (int q = 0; q < AC; ++q) {
        const bool pos = wy[q] >= T(0);
        const T lf = wy[q] * (pos ? l[q] : c[q]);
        const T rf = wy[q] * (pos ? c[q] : r[q]);
        div[q] = (rf - lf) * rdy;
    }
    lds<T, AC>(Gz + rg.at(gy, gz) * AC, c);
    lds<T, AC>(gz > 0 ? Gz + rg.at(gy, gz - 1) * AC : X + rx.at(gy, 0) * AC, l);
    lds<T, AC>(gz < Nz ? Gz + rg.at(gy, gz + 1) * AC : X + rx.at(gy, Nz) * AC, r);
#pragma unroll
    for (int q = 0; q < AC; ++q) {
        const bool pos = wz[q] >= T(0);
        const T lf = wz[q] * (pos ? l[q] : c[q]);
        const T rf = wz[q] * (pos ? c[q] : r[q]);
        div[q] += (rf - lf) * rdz;
    }
}

// One block = one energy group, AC consecutive angles, one tile of output
// positions; one thread per position with all AC angles in registers.
// Shared memory holds F over the tile plus a 4-cell halo (overwritten in
// place by H = F - dt/2 div F on the tile once it is no longer read), the
// face values (3-cell halo, reused for the predictor's faces) and the
// predictor (2-cell halo).  Every slope is evaluated once per cell and
// direction.
template <typename T, int AC>
__global__ void __launch_bounds__(256) transport_kernel(TransportArgs<T> a, int tiles_y, int tiles_z, int n_chunks) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int b = blockIdx.x;
    const int tyi = b % tiles_y;
    b /= tiles_y;
    const int tzi = b % tiles_z;
    b /= tiles_z;
    const int chunk = b % n_chunks;
    const int ek = b / n_chunks;
    const int Ny = a.Ny, Nz = a.Nz, Ny1 = a.Ny + 1, Nz1 = a.Nz + 1, NA = a.NA;
    const Rect t{tyi * a.tile_y, min(tyi * a.tile_y + a.tile_y, Ny1), tzi * a.tile_z, min(tzi * a.tile_z + a.tile_z, Nz1)};
    const Rect r1 = t.grow(1, Ny1, Nz1), r2 = t.grow(2, Ny1, Nz1), r3 = t.grow(3, Ny1, Nz1), r4 = t.grow(4, Ny1, Nz1);
    T* Fs = reinterpret_cast<T*>(smem_raw);
    T* Gy = Fs + r4.n() * AC;
    T* Gz = Gy + r3.n() * AC;
    T* Ps = Gz + r3.n() * AC;
    const int a0 = chunk * AC;
    const size_t plane = static_cast<size_t>(ek) * Ny1 * Nz1 * NA + a0;
    const T* __restrict__ in = a.in + plane;
    T* __restrict__ out = a.out + plane;
    const T dt = a.dt, rdy = T(1) / a.dy, rdz = T(1) / a.dz, hdt = T(0.5) * a.dt;
    const bool full = a0 + AC <= NA;
    T wy[AC], wz[AC], hy[AC], hz[AC];
#pragma unroll
    for (int q = 0; q < AC; ++q) {
        const int ang = min(a0 + q, NA - 1);
        wy[q] = a.omega[2 * ang];
        wz[q] = a.omega[2 * ang + 1];
        hy[q] = wy[q] >= T(0) ? T(0.5) : T(-0.5);
        hz[q] = wz[q] >= T(0) ? T(0.5) : T(-0.5);
    }
    {
        const float inv_w = 1.0f / r4.w();
        for (int p = threadIdx.x; p < r4.n(); p += blockDim.x) {
            int gy, gz;
            rect_pos(r4, p, inv_w, gy, gz);
            const T* src = in + (static_cast<size_t>(gz) * Ny1 + gy) * NA;
            T v[AC];
#pragma unroll
            for (int q = 0; q < AC; ++q) v[q] = (full || a0 + q < NA) ? src[q] : T(0);
            sts<T, AC>(Fs + p * AC, v);
        }
    }
    __syncthreads();
    build_faces<T, AC>(Fs, r4, Gy, Gz, r3, r3, Ny, Nz, hy, hz);
    __syncthreads();
    {  // predictor over r2; H over the tile into F's own slots (each thread reads F only at its position)
        const float inv_w = 1.0f / r2.w();
        for (int p = threadIdx.x; p < r2.n(); p += blockDim.x) {
            int gy, gz;
            rect_pos(r2, p, inv_w, gy, gz);
            T d[AC], f[AC], v[AC];
            face_divergence<T, AC>(Fs, r4, Gy, Gz, r3, gy, gz, Ny, Nz, wy, wz, rdy, rdz, d);
            T* fp = Fs + r4.at(gy, gz) * AC;
            lds<T, AC>(fp, f);
#pragma unroll
            for (int q = 0; q < AC; ++q) {
                const T x = f[q] - dt * d[q];
                v[q] = a.preserve_sign ? x : max(x, T(0));
            }
            sts<T, AC>(Ps + p * AC, v);
            if (gy >= t.y0 && gy < t.y1 && gz >= t.z0 && gz < t.z1) {
#pragma unroll
                for (int q = 0; q < AC; ++q) v[q] = f[q] - hdt * d[q];
                sts<T, AC>(fp, v);
            }
        }
    }
    __syncthreads();
    build_faces<T, AC>(Ps, r2, Gy, Gz, r3, r1, Ny, Nz, hy, hz);
    __syncthreads();
    {  // corrector over the tile
        const float inv_w = 1.0f / t.w();
        for (int p = threadIdx.x; p < t.n(); p += blockDim.x) {
            int gy, gz;
            rect_pos(t, p, inv_w, gy, gz);
            T d[AC], h[AC];
            face_divergence<T, AC>(Ps, r2, Gy, Gz, r3, gy, gz, Ny, Nz, wy, wz, rdy, rdz, d);
            lds<T, AC>(Fs + r4.at(gy, gz) * AC, h);
            T* dst = out + (static_cast<size_t>(gz) * Ny1 + gy) * NA;
#pragma unroll
            for (int q = 0; q < AC; ++q) {
                const T x = h[q] - hdt * d[q];
                if (full || a0 + q < NA) dst[q] = a.preserve_sign ? x : max(x, T(0));
            }
        }
    }
}

// Shared memory of one transport block for a tile of ty x tz positions.
size_t transport_smem(int Ny1, int Nz1, int ty, int tz, int ac, size_t elem) {
    auto n = [&](int h) {
        return static_cast<size_t>(std::min(Ny1, ty + 2 * h)) * std::min(Nz1, tz + 2 * h);
    };
    return (n(4) + 2 * n(3) + n(2)) * ac * elem;
}

template <typename T, int AC>
static cudaError_t launch_transport_ac(const TransportArgs<T>& a, cudaStream_t s) {
    const int Ny1 = a.Ny + 1, Nz1 = a.Nz + 1;
    const int tiles_y = (Ny1 + a.tile_y - 1) / a.tile_y, tiles_z = (Nz1 + a.tile_z - 1) / a.tile_z;
    const int n_chunks = (a.NA + AC - 1) / AC;
    const size_t smem = transport_smem(Ny1, Nz1, a.tile_y, a.tile_z, AC, sizeof(T));
    auto kern = transport_kernel<T, AC>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const long long blocks = static_cast<long long>(a.Ng) * n_chunks * tiles_y * tiles_z;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    // one thread per position of the largest staged region, in whole warps, at most 256
    const int npos = std::min(Ny1, a.tile_y + 8) * std::min(Nz1, a.tile_z + 8);
    const int rounds = (npos + 255) / 256;
    const int threads = std::min(256, ((npos + rounds - 1) / rounds + 31) / 32 * 32);
    kern<<<static_cast<unsigned>(blocks), threads, smem, s>>>(a, tiles_y, tiles_z, n_chunks);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_transport(const TransportArgs<T>& a, int ang_chunk, cudaStream_t s) {
    switch (ang_chunk) {
        case 4: return launch_transport_ac<T, 4>(a, s);
        case 8: return launch_transport_ac<T, 8>(a, s);
        case 16: return launch_transport_ac<T, 16>(a, s);
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
