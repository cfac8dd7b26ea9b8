// Depth-step kernels: eq15 energy sweep (with fused IDD partials), MUSCL
// predictor-corrector transport, separable DST-I angular diffusion, IDD
// finalisation, beam initialisation and conversions.
//
// State layout (HBM): index = (ek * nyz + pos) * NA + ang, ang fastest, the
// index order of the reference (bfpm_solver.cu:1996).  Every kernel walks
// ang with consecutive threads, so global accesses are coalesced.

#include "common.cuh"
#include "async_copy.cuh"

#include <cuda_bf16.h>

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <type_traits>
#include <utility>

namespace bfpn {

template <int V>
using IntC = std::integral_constant<int, V>;

cudaError_t allow_dynamic_smem(const void* func, size_t need) {
    static std::mutex m;
    static std::map<std::pair<const void*, int>, size_t> limit;  // (function, device) -> bytes allowed
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(m);
    auto it = limit.find({func, dev});
    if (it == limit.end()) {
        cudaFuncAttributes fa{};
        int optin = 0;
        if ((e = cudaFuncGetAttributes(&fa, func)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess) return e;
        const size_t allow = optin > static_cast<int>(fa.sharedSizeBytes) ? optin - fa.sharedSizeBytes : 0;
        if ((e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(allow))) !=
            cudaSuccess)
            return e;
        it = limit.emplace(std::make_pair(func, dev), allow).first;
    }
    return need <= it->second ? cudaSuccess : cudaErrorInvalidValue;
}

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
constexpr int kEnergyLanesPerThread = 2;

// One group of the eq15 / legacy recursion for one lane (energyDgCnKernel,
// energy_solver.cu:88-159): Fg, fg old values of group ek, sg its source,
// Fn the old psi^1 of group ek-1 (straggling), F_hi_old / f_hi_old the old
// values of group ek+1 and next_F / next_f its new values.
template <int MODE>
__device__ __forceinline__ void energy_lane_update(const double* __restrict__ c, int ek, double Fg, double fg,
                                                   double sg, double Fn, double F_hi_old, double f_hi_old,
                                                   double next_F, double next_f, double& Fv, double& fv) {
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
        const double rhs = __ldg(c + EC_R_F) * fg + __ldg(c + EC_R_UP) * up + __ldg(c + EC_R_CUR) * cur +
                           __ldg(c + EC_R_FG) * Fg - __ldg(c + EC_A) * common + __ldg(c + EC_R_HI) * hi_delta;
        fv = rhs * __ldg(c + EC_INV_COE);
        Fv = __ldg(c + EC_F_FROM_F) * fv + __ldg(c + EC_INV_F) * common + __ldg(c + EC_F_FROM_HI) * hi_delta;
    }
}

// The sweep of block `bid` of one beam's lanes (the kernels below map their
// blocks onto it: one beam, or the slots of a bundle).
// The eq15 constants of one group held in registers (loaded a group ahead by
// the ring sweep, so their loads are off the recursion's critical path), and
// the eq15 update of energy_lane_update from them: the same operations in the
// same order.
struct Eq15Coef {
    double c_up, c_cur, c_f, r_f, r_up, r_cur, r_fg, a, r_hi, inv_coe, f_from_f, inv_f, f_from_hi;
    double s_hi, s_lo, s_g;  // straggling
    double d0, d1;           // dose weights of psi^1, psi^2
};

template <int MODE>
__device__ __forceinline__ Eq15Coef load_eq15_coef(const double* __restrict__ c, const double* __restrict__ dc,
                                                   bool dose) {
    Eq15Coef k;
    k.c_up = __ldg(c + EC_C_UP);
    k.c_cur = __ldg(c + EC_C_CUR);
    k.c_f = __ldg(c + EC_C_F);
    k.r_f = __ldg(c + EC_R_F);
    k.r_up = __ldg(c + EC_R_UP);
    k.r_cur = __ldg(c + EC_R_CUR);
    k.r_fg = __ldg(c + EC_R_FG);
    k.a = __ldg(c + EC_A);
    k.r_hi = __ldg(c + EC_R_HI);
    k.inv_coe = __ldg(c + EC_INV_COE);
    k.f_from_f = __ldg(c + EC_F_FROM_F);
    k.inv_f = __ldg(c + EC_INV_F);
    k.f_from_hi = __ldg(c + EC_F_FROM_HI);
    k.s_hi = k.s_lo = k.s_g = 0.0;
    if (MODE == EMODE_EQ15_STRAG) {
        k.s_hi = __ldg(c + EC_S_HI);
        k.s_lo = __ldg(c + EC_S_LO);
        k.s_g = __ldg(c + EC_S_G);
    }
    k.d0 = dose ? __ldg(dc) : 0.0;
    k.d1 = dose ? __ldg(dc + 1) : 0.0;
    return k;
}

template <int MODE>
__device__ __forceinline__ void eq15_update(const Eq15Coef& k, int ek, double Fg, double fg, double sg, double Fn,
                                            double F_hi_old, double f_hi_old, double next_F, double next_f,
                                            double& Fv, double& fv) {
    const double up = F_hi_old - f_hi_old;
    const double cur = Fg - fg;
    double common = k.c_up * up + k.c_cur * cur + k.c_f * Fg + sg;
    if (MODE == EMODE_EQ15_STRAG) {
        const double Flo = (ek > 0) ? Fn : 0.0;
        common += k.s_hi * F_hi_old + k.s_lo * Flo - k.s_g * Fg;
    }
    const double hi_delta = next_F - next_f;
    const double rhs = k.r_f * fg + k.r_up * up + k.r_cur * cur + k.r_fg * Fg - k.a * common + k.r_hi * hi_delta;
    fv = rhs * k.inv_coe;
    Fv = k.f_from_f * fv + k.inv_f * common + k.f_from_hi * hi_delta;
}

template <int MODE, typename T, int LPT, int D>
__device__ __forceinline__ void energy_body(const EnergyArgs<T>& a, long long bid) {
    // D: groups prefetched ahead of use
    const long long L = a.lanes;
    const int Ng = a.Ng;
    long long lane[LPT];
    bool ok[LPT];
#pragma unroll
    for (int j = 0; j < LPT; ++j) {
        lane[j] = bid * blockDim.x * LPT + threadIdx.x + j * blockDim.x;
        ok[j] = lane[j] < L;
    }
    const T* __restrict__ sp = a.src;
    // ring of the next D groups' old values for each lane
    T rF[D][LPT], rf[D][LPT], rs[D][LPT];
#pragma unroll
    for (int k = 0; k < D; ++k)
#pragma unroll
        for (int j = 0; j < LPT; ++j) {
            const int e = Ng - 1 - k;
            const bool in = ok[j] && e >= 0;
            rF[k][j] = in ? a.F[e * L + lane[j]] : T(0);
            rf[k][j] = in ? a.f[e * L + lane[j]] : T(0);
            rs[k][j] = (in && sp) ? sp[e * L + lane[j]] : T(0);
        }
    double F_hi_old[LPT], f_hi_old[LPT], next_F[LPT], next_f[LPT], w_pos[LPT], acc = 0.0, accp = 0.0;
#pragma unroll
    for (int j = 0; j < LPT; ++j) {
        F_hi_old[j] = f_hi_old[j] = next_F[j] = next_f[j] = 0.0;
        w_pos[j] = 1.0;
        if (a.partials && a.trapezoidal && ok[j]) {
            const int pos = static_cast<int>((lane[j] + a.lane0) / a.NA);
            const int iy = pos % (a.Ny + 1), iz = pos / (a.Ny + 1);
            if (iy == 0 || iy == a.Ny) w_pos[j] *= 0.5;
            if (iz == 0 || iz == a.Nz) w_pos[j] *= 0.5;
        }
    }
    for (int base = Ng - 1; base >= 0; base -= D)
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const int ek = base - k;
        if (ek < 0) break;
        const double* __restrict__ c = a.coef + ek * kEnergyCoef;
        const double* __restrict__ dc = a.dose_coef + 2 * ek;
        const int ep = ek - D;  // the group that refills this slot
#pragma unroll
        for (int j = 0; j < LPT; ++j) {
            const double Fg = static_cast<double>(rF[k][j]), fg = static_cast<double>(rf[k][j]),
                         sg = static_cast<double>(rs[k][j]);
            if (ep >= 0 && ok[j]) {
                rF[k][j] = a.F[ep * L + lane[j]];
                rf[k][j] = a.f[ep * L + lane[j]];
                if (sp) rs[k][j] = sp[ep * L + lane[j]];
            }
            // old value of group ek-1 (straggling): the next slot, or the refill of slot 0
            const double Fn = static_cast<double>(rF[(k + 1) % D][j]);
            double Fv, fv;
            energy_lane_update<MODE>(c, ek, Fg, fg, sg, Fn, F_hi_old[j], f_hi_old[j], next_F[j], next_f[j], Fv, fv);
            const T Fs = static_cast<T>(Fv), fs = static_cast<T>(fv);
            if (ok[j]) {
                a.F[ek * L + lane[j]] = Fs;
                a.f[ek * L + lane[j]] = fs;
                if (a.partials) {
                    acc += w_pos[j] * (__ldg(dc) * static_cast<double>(Fs) + __ldg(dc + 1) * static_cast<double>(fs));
                    accp += static_cast<double>(fs);
                }
            }
            F_hi_old[j] = Fg;
            f_hi_old[j] = fg;
            next_F[j] = Fv;
            next_f[j] = fv;
        }
    }
    if (a.partials) {
        __shared__ double red[2][32];
        for (int o = 16; o > 0; o >>= 1) {
            acc += __shfl_down_sync(0xffffffffu, acc, o);
            accp += __shfl_down_sync(0xffffffffu, accp, o);
        }
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        if (l == 0) {
            red[0][w] = acc;
            red[1][w] = accp;
        }
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
                a.partials[2 * bid] = acc;
                a.partials[2 * bid + 1] = accp;
            }
        }
    }
}

template <int MODE, typename T, int LPT, int D = 4, int NTH = 128, int MINB = (sizeof(T) == 4 ? 5 : 4)>
__global__ void __launch_bounds__(NTH, MINB) energy_kernel(EnergyArgs<T> a) {
    energy_body<MODE, T, LPT, D>(a, blockIdx.x);
}

template <int MODE, int LPT, int D = 4, int NTH = 128, int MINB = 5>
__global__ void __launch_bounds__(NTH, MINB) energy_slots_kernel(const EnergyArgs<float>* __restrict__ args,
                                                                  const int* __restrict__ begin, int nslots) {
    const int s = find_slot(begin, nslots, blockIdx.x);
    energy_body<MODE, float, LPT, D>(args[s], blockIdx.x - __ldg(begin + s));
}

// Float state, lanes a multiple of 4: each thread sweeps 4 consecutive lanes
// and keeps its own ring of the next groups' old values in shared memory,
// filled by 16-byte cp.async copies (no registers held by the prefetch, no
// block barrier: a thread only reads what it copied).  Slot i % D holds group
// Ng-1-i; the slot consumed in one iteration is refilled in the next, so up
// to D-2 groups are in flight ahead of the one in use.  Same update and IDD
// partials as energy_kernel.
constexpr int kEnergyRing = 8, kEnergyRingThreads = 64;

template <int MODE, int D, int NTH>
__device__ __forceinline__ void energy_ring_body(const EnergyArgs<float>& a, long long bid) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* ring = reinterpret_cast<float4*>(smem_raw);  // [D][3][NTH]
    const long long L = a.lanes;
    const int Ng = a.Ng, tid = threadIdx.x;
    const long long lane0 = (bid * NTH + tid) * 4;
    const bool ok = lane0 < L;  // L % 4 == 0: the 4 lanes are all in or all out
    const float* __restrict__ sp = a.src;
    auto slot = [&](int k, int arr) { return ring + (k * 3 + arr) * NTH + tid; };
    auto fill = [&](int i) {  // group Ng-1-i into slot i % D, one commit group per call
        const int e = Ng - 1 - i;
        if (ok && e >= 0) {
            const size_t off = static_cast<size_t>(e) * L + lane0;
            cp_async16(slot(i % D, 0), a.F + off, true);
            cp_async16(slot(i % D, 1), a.f + off, true);
            if (sp) cp_async16(slot(i % D, 2), sp + off, true);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    for (int i = 0; i < D; ++i) fill(i);
    double F_hi_old[4], f_hi_old[4], next_F[4], next_f[4], w_pos[4], acc = 0.0, accp = 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        F_hi_old[j] = f_hi_old[j] = next_F[j] = next_f[j] = 0.0;
        w_pos[j] = 1.0;
        if (a.partials && a.trapezoidal && ok) {
            const int pos = static_cast<int>((lane0 + j + a.lane0) / a.NA);
            const int iy = pos % (a.Ny + 1), iz = pos / (a.Ny + 1);
            if (iy == 0 || iy == a.Ny) w_pos[j] *= 0.5;
            if (iz == 0 || iz == a.Nz) w_pos[j] *= 0.5;
        }
    }
    constexpr bool kStrag = MODE == EMODE_EQ15_STRAG;
    const bool dose = a.partials != nullptr;
    // group Ng-1-i's constants in K[i % 2]; iteration i loads the next
    // group's into the other slot.  Two iterations per trip keep the slots
    // fixed registers instead of a copy of the set per group.
    Eq15Coef K[2];
    K[0] = load_eq15_coef<MODE>(a.coef + (Ng - 1) * kEnergyCoef, a.dose_coef + 2 * (Ng - 1), dose);
    auto iter = [&](auto Rc, int i) {
        constexpr int R = decltype(Rc)::value;
        const int ek = Ng - 1 - i;
        if (ek < 0) return;
        const Eq15Coef& kc = K[R];
        if (ek > 0) K[R ^ 1] = load_eq15_coef<MODE>(a.coef + (ek - 1) * kEnergyCoef, a.dose_coef + 2 * (ek - 1), dose);
        // groups 0 .. i (and i+1 for straggling) have landed
        if (kStrag) asm volatile("cp.async.wait_group %0;" ::"n"(D - 3) : "memory");
        else asm volatile("cp.async.wait_group %0;" ::"n"(D - 2) : "memory");
        const float4 vF = *slot(i % D, 0), vf = *slot(i % D, 1);
        const float4 vs = sp ? *slot(i % D, 2) : make_float4(0.f, 0.f, 0.f, 0.f);
        float4 vn = make_float4(0.f, 0.f, 0.f, 0.f);
        if (kStrag && ek > 0) vn = *slot((i + 1) % D, 0);
        if (i > 0) fill(i - 1 + D);  // the slot read in the previous iteration
        const float Fa[4] = {vF.x, vF.y, vF.z, vF.w}, fa[4] = {vf.x, vf.y, vf.z, vf.w};
        const float sa[4] = {vs.x, vs.y, vs.z, vs.w}, na[4] = {vn.x, vn.y, vn.z, vn.w};
        float Fo[4], fo[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double Fg = Fa[j], fg = fa[j];
            double Fv, fv;
            eq15_update<MODE>(kc, ek, Fg, fg, static_cast<double>(sa[j]), static_cast<double>(na[j]), F_hi_old[j],
                              f_hi_old[j], next_F[j], next_f[j], Fv, fv);
            Fo[j] = static_cast<float>(Fv);
            fo[j] = static_cast<float>(fv);
            if (dose && ok) {
                acc += w_pos[j] * (kc.d0 * static_cast<double>(Fo[j]) + kc.d1 * static_cast<double>(fo[j]));
                accp += static_cast<double>(fo[j]);
            }
            F_hi_old[j] = Fg;
            f_hi_old[j] = fg;
            next_F[j] = Fv;
            next_f[j] = fv;
        }
        if (ok) {
            const size_t off = static_cast<size_t>(ek) * L + lane0;
            *reinterpret_cast<float4*>(a.F + off) = make_float4(Fo[0], Fo[1], Fo[2], Fo[3]);
            *reinterpret_cast<float4*>(a.f + off) = make_float4(fo[0], fo[1], fo[2], fo[3]);
        }
    };
#pragma unroll 1
    for (int i = 0; i < Ng; i += 2) {
        iter(IntC<0>(), i);
        iter(IntC<1>(), i + 1);
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    if (a.partials) {
        __shared__ double red[2][NTH / 32];
        for (int o = 16; o > 0; o >>= 1) {
            acc += __shfl_down_sync(0xffffffffu, acc, o);
            accp += __shfl_down_sync(0xffffffffu, accp, o);
        }
        const int w = tid >> 5, l = tid & 31;
        if (l == 0) {
            red[0][w] = acc;
            red[1][w] = accp;
        }
        __syncthreads();
        if (tid == 0) {
            double s0 = 0.0, s1 = 0.0;
            for (int k = 0; k < NTH / 32; ++k) {
                s0 += red[0][k];
                s1 += red[1][k];
            }
            a.partials[2 * bid] = s0;
            a.partials[2 * bid + 1] = s1;
        }
    }
}

template <int MODE, int D, int NTH>
__global__ void __launch_bounds__(NTH) energy_ring_kernel(EnergyArgs<float> a) {
    energy_ring_body<MODE, D, NTH>(a, blockIdx.x);
}

template <int MODE, int D, int NTH>
__global__ void __launch_bounds__(NTH) energy_ring_slots_kernel(const EnergyArgs<float>* __restrict__ args,
                                                                const int* __restrict__ begin, int nslots) {
    const int s = find_slot(begin, nslots, blockIdx.x);
    energy_ring_body<MODE, D, NTH>(args[s], blockIdx.x - __ldg(begin + s));
}

int energy_ring_grid(long long lanes) {
    const long long per_block = 4LL * kEnergyRingThreads;
    return static_cast<int>((lanes + per_block - 1) / per_block);
}

cudaError_t launch_energy_ring(const EnergyArgs<float>& a, cudaStream_t s) {
    if (a.lanes % 4 != 0 || a.mode == EMODE_LEGACY) return cudaErrorNotSupported;
    constexpr int D = kEnergyRing, NTH = kEnergyRingThreads;
    const size_t smem = static_cast<size_t>(D) * 3 * NTH * sizeof(float4);
    const int grid = energy_ring_grid(a.lanes);
    if (a.mode == EMODE_EQ15) energy_ring_kernel<EMODE_EQ15, D, NTH><<<grid, NTH, smem, s>>>(a);
    else energy_ring_kernel<EMODE_EQ15_STRAG, D, NTH><<<grid, NTH, smem, s>>>(a);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Fused primary energy half-steps: the closing E1/2 of step n and the opening
// E1/2 of step n+1 in one sweep over the groups (high -> low).  The opening
// sweep's update of group g needs the closing result of groups g and g-1
// (straggling) and its own results for g+1, so it runs one group behind the
// closing sweep, its carried values in registers: iteration i applies the
// closing update to group ek = Ng-1-i and the opening update to group ek+1.
// Each update is energy_ring_kernel's, on the same inputs -- the midpoint
// value is rounded to float as the separate passes store it -- so the state
// equals the two passes' bit for bit on the grids tested, except a few values
// far below the peak, which may come out one float rounding step apart (on a
// 35 x 35, 12-group grid: values 1e-8 below the peak, 4.6e-16 of it).  The closing pass's IDD partials are those of the
// closing ring pass.  At the midpoint the source groups' values
// go to the angular contraction's operand (split bf16), which removes that
// operand's own pass over the primary.
// ---------------------------------------------------------------------------
template <int MODE, int D, int NTH>
__global__ void __launch_bounds__(NTH) energy_fused_kernel(EnergyFusedArgs A) {
    const EnergyArgs<float>& a = A.e;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* ring = reinterpret_cast<float4*>(smem_raw);  // [D][2][NTH]
    const long long L = a.lanes;
    const int Ng = a.Ng, tid = threadIdx.x;
    const long long bid = blockIdx.x;
    const long long lane0 = (bid * NTH + tid) * 4;
    const bool ok = lane0 < L;  // L % 4 == 0: the 4 lanes are all in or all out
    auto slot = [&](int k, int arr) { return ring + (k * 2 + arr) * NTH + tid; };
    auto fill = [&](int i) {  // group Ng-1-i into slot i % D, one commit group per call
        const int e = Ng - 1 - i;
        if (ok && e >= 0) {
            const size_t off = static_cast<size_t>(e) * L + lane0;
            cp_async16(slot(i % D, 0), a.F + off, true);
            cp_async16(slot(i % D, 1), a.f + off, true);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    for (int i = 0; i < D; ++i) fill(i);
    // closing sweep: old values and new values of the group above; opening
    // sweep: midpoint values and new values of the group above its own
    double cFo[4], cfo[4], cFn[4], cfn[4], oFo[4], ofo[4], oFn[4], ofn[4], w_pos[4], acc = 0.0, accp = 0.0;
    float mF[4], mf[4];  // midpoint of group ek+1
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        cFo[j] = cfo[j] = cFn[j] = cfn[j] = oFo[j] = ofo[j] = oFn[j] = ofn[j] = 0.0;
        mF[j] = mf[j] = 0.f;
        w_pos[j] = 1.0;
        if (a.partials && a.trapezoidal && ok) {
            const int pos = static_cast<int>((lane0 + j) / a.NA);
            const int iy = pos % (a.Ny + 1), iz = pos / (a.Ny + 1);
            if (iy == 0 || iy == a.Ny) w_pos[j] *= 0.5;
            if (iz == 0 || iz == a.Nz) w_pos[j] *= 0.5;
        }
    }
    // this thread's place in the source operand: position p, angles k0 .. k0+3 of chunk kc
    const int p = ok ? static_cast<int>(lane0 / a.NA) : 0, k0 = ok ? static_cast<int>(lane0 % a.NA) : 0;
    constexpr size_t kPart = 128 * 16 * 2;  // one (hi or lo) 128 x 16 bf16 tile
    const size_t a_tile = (static_cast<size_t>(p >> 6) * A.nk + (k0 >> 4)) * 2 * kPart;
    const size_t a_off1 = umma_kmajor_offset(p & 63, k0 & 15, 128), a_off2 = umma_kmajor_offset(64 + (p & 63), k0 & 15, 128);
    const size_t a_group = static_cast<size_t>(A.n_mt) * A.nk * 2 * kPart;
    auto put = [&](size_t off, float x0, float x1, float x2, float x3) {  // 4 values: hi, then lo
        const __nv_bfloat162 h01 = __floats2bfloat162_rn(x0, x1), h23 = __floats2bfloat162_rn(x2, x3);
        const __nv_bfloat162 l01 = __floats2bfloat162_rn(x0 - __low2float(h01), x1 - __high2float(h01));
        const __nv_bfloat162 l23 = __floats2bfloat162_rn(x2 - __low2float(h23), x3 - __high2float(h23));
        uint2 hv, lv;
        hv.x = *reinterpret_cast<const uint32_t*>(&h01);
        hv.y = *reinterpret_cast<const uint32_t*>(&h23);
        lv.x = *reinterpret_cast<const uint32_t*>(&l01);
        lv.y = *reinterpret_cast<const uint32_t*>(&l23);
        *reinterpret_cast<uint2*>(A.ablob + off) = hv;
        *reinterpret_cast<uint2*>(A.ablob + off + kPart) = lv;
    };
    constexpr bool kStrag = MODE == EMODE_EQ15_STRAG;
    const bool dose = a.partials != nullptr;
    Eq15Coef k_next = load_eq15_coef<MODE>(a.coef + (Ng - 1) * kEnergyCoef, a.dose_coef + 2 * (Ng - 1), dose);
    Eq15Coef k_up = k_next;  // constants of group ek+1 (the opening update's group)
    for (int i = 0; i <= Ng; ++i) {
        const int ek = Ng - 1 - i;
        float nF[4] = {0.f, 0.f, 0.f, 0.f}, nf[4] = {0.f, 0.f, 0.f, 0.f};  // midpoint of group ek
        Eq15Coef kc = k_up;
        if (ek >= 0) {
            // closing update of group ek
            kc = k_next;
            if (ek > 0) k_next = load_eq15_coef<MODE>(a.coef + (ek - 1) * kEnergyCoef, a.dose_coef + 2 * (ek - 1), dose);
            if (kStrag) asm volatile("cp.async.wait_group %0;" ::"n"(D - 3) : "memory");
            else asm volatile("cp.async.wait_group %0;" ::"n"(D - 2) : "memory");
            const float4 vF = *slot(i % D, 0), vf = *slot(i % D, 1);
            float4 vn = make_float4(0.f, 0.f, 0.f, 0.f);
            if (kStrag && ek > 0) vn = *slot((i + 1) % D, 0);
            if (i > 0) fill(i - 1 + D);  // the slot read in the previous iteration
            const float Fa[4] = {vF.x, vF.y, vF.z, vF.w}, fa[4] = {vf.x, vf.y, vf.z, vf.w};
            const float na[4] = {vn.x, vn.y, vn.z, vn.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const double Fg = Fa[j], fg = fa[j];
                double Fv, fv;
                eq15_update<MODE>(kc, ek, Fg, fg, 0.0, static_cast<double>(na[j]), cFo[j], cfo[j], cFn[j], cfn[j],
                                  Fv, fv);
                nF[j] = static_cast<float>(Fv);
                nf[j] = static_cast<float>(fv);
                if (dose && ok) {
                    acc += w_pos[j] * (kc.d0 * static_cast<double>(nF[j]) + kc.d1 * static_cast<double>(nf[j]));
                    accp += static_cast<double>(nf[j]);
                }
                cFo[j] = Fg;
                cfo[j] = fg;
                cFn[j] = Fv;
                cfn[j] = fv;
            }
            const int gz = A.ablob ? __ldg(A.gmap + ek) : -1;
            if (ok && gz >= 0) {
                const size_t base = static_cast<size_t>(gz) * a_group + a_tile;
                put(base + a_off1, fmaxf(nF[0], 0.f), fmaxf(nF[1], 0.f), fmaxf(nF[2], 0.f), fmaxf(nF[3], 0.f));
                put(base + a_off2, nf[0], nf[1], nf[2], nf[3]);
            }
        }
        if (ek + 1 <= Ng - 1) {
            // opening update of group ek+1 from the midpoint: its value mF/mf,
            // group ek's (straggling) nF, the group above's oFo/oFn
            const int eo = ek + 1;
            float Fo[4], fo[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const double Fg = mF[j], fg = mf[j];
                double Fv, fv;
                eq15_update<MODE>(k_up, eo, Fg, fg, 0.0, static_cast<double>(nF[j]), oFo[j], ofo[j], oFn[j], ofn[j],
                                  Fv, fv);
                Fo[j] = static_cast<float>(Fv);
                fo[j] = static_cast<float>(fv);
                oFo[j] = Fg;
                ofo[j] = fg;
                oFn[j] = Fv;
                ofn[j] = fv;
            }
            if (ok) {
                const size_t off = static_cast<size_t>(eo) * L + lane0;
                *reinterpret_cast<float4*>(a.F + off) = make_float4(Fo[0], Fo[1], Fo[2], Fo[3]);
                *reinterpret_cast<float4*>(a.f + off) = make_float4(fo[0], fo[1], fo[2], fo[3]);
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            mF[j] = nF[j];
            mf[j] = nf[j];
        }
        k_up = kc;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    if (a.partials) {
        __shared__ double red[2][NTH / 32];
        for (int o = 16; o > 0; o >>= 1) {
            acc += __shfl_down_sync(0xffffffffu, acc, o);
            accp += __shfl_down_sync(0xffffffffu, accp, o);
        }
        const int w = tid >> 5, l = tid & 31;
        if (l == 0) {
            red[0][w] = acc;
            red[1][w] = accp;
        }
        __syncthreads();
        if (tid == 0) {
            double s0 = 0.0, s1 = 0.0;
            for (int k = 0; k < NTH / 32; ++k) {
                s0 += red[0][k];
                s1 += red[1][k];
            }
            a.partials[2 * bid] = s0;
            a.partials[2 * bid + 1] = s1;
        }
    }
}

bool energy_fused_supported(long long lanes, int mode, int NA) {
    return lanes % 4 == 0 && NA % 4 == 0 && mode != EMODE_LEGACY;
}

cudaError_t launch_energy_fused(const EnergyFusedArgs& A, cudaStream_t s) {
    const EnergyArgs<float>& a = A.e;
    if (!energy_fused_supported(a.lanes, a.mode, a.NA) || a.src || a.lane0 != 0) return cudaErrorNotSupported;
    constexpr int D = kEnergyRing, NTH = kEnergyRingThreads;
    const size_t smem = static_cast<size_t>(D) * 2 * NTH * sizeof(float4);
    const int grid = energy_ring_grid(a.lanes);
    if (a.mode == EMODE_EQ15) energy_fused_kernel<EMODE_EQ15, D, NTH><<<grid, NTH, smem, s>>>(A);
    else energy_fused_kernel<EMODE_EQ15_STRAG, D, NTH><<<grid, NTH, smem, s>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_energy_slots(const EnergyArgs<float>* args, const int* begin, int nslots, int blocks, int mode,
                                bool ring, int block, cudaStream_t s) {
    if (nslots <= 0 || blocks <= 0) return cudaSuccess;
    if (ring) {
        if (mode == EMODE_LEGACY) return cudaErrorNotSupported;
        constexpr int D = kEnergyRing, NTH = kEnergyRingThreads;
        const size_t smem = static_cast<size_t>(D) * 3 * NTH * sizeof(float4);
        if (mode == EMODE_EQ15) energy_ring_slots_kernel<EMODE_EQ15, D, NTH><<<blocks, NTH, smem, s>>>(args, begin, nslots);
        else energy_ring_slots_kernel<EMODE_EQ15_STRAG, D, NTH><<<blocks, NTH, smem, s>>>(args, begin, nslots);
        return cudaGetLastError();
    }
    if (block != 128) return cudaErrorNotSupported;
    constexpr int LPT = kEnergyLanesPerThread;
    switch (mode) {
        case EMODE_EQ15: energy_slots_kernel<EMODE_EQ15, LPT><<<blocks, 128, 0, s>>>(args, begin, nslots); break;
        case EMODE_EQ15_STRAG:
            energy_slots_kernel<EMODE_EQ15_STRAG, LPT><<<blocks, 128, 0, s>>>(args, begin, nslots);
            break;
        default: energy_slots_kernel<EMODE_LEGACY, LPT><<<blocks, 128, 0, s>>>(args, begin, nslots); break;
    }
    return cudaGetLastError();
}

int energy_grid(long long lanes, int block) {
    const long long per_block = static_cast<long long>(block) * kEnergyLanesPerThread;
    return static_cast<int>((lanes + per_block - 1) / per_block);
}

template <typename T>
cudaError_t launch_energy(const EnergyArgs<T>& a, int block, cudaStream_t s) {
    constexpr int LPT = kEnergyLanesPerThread;
    if constexpr (sizeof(T) == 4) {
        // planes of at least 2^20 lanes fill the GPU with 64-thread ring blocks
        // (4 lanes a thread); smaller ones keep more threads per SM with the
        // register ring.  Same partial count: 4 * 64 lanes per block = 2 * 128.
        if (a.lanes >= (1LL << 20) && a.lanes % 4 == 0 && a.mode != EMODE_LEGACY &&
            block * LPT == 4 * kEnergyRingThreads)
            return launch_energy_ring(a, s);
    }
    const int grid = energy_grid(a.lanes, block);
    switch (a.mode) {
        case EMODE_EQ15: energy_kernel<EMODE_EQ15, T, LPT><<<grid, block, 0, s>>>(a); break;
        case EMODE_EQ15_STRAG: energy_kernel<EMODE_EQ15_STRAG, T, LPT><<<grid, block, 0, s>>>(a); break;
        default: energy_kernel<EMODE_LEGACY, T, LPT><<<grid, block, 0, s>>>(a); break;
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Lite-memory primary step (litePrimaryEnergyStepKernel, bfpm_solver.cu:593-620):
// psi^1 only, first-order upwind in energy with catastrophic attenuation,
// groups swept from Ng-1 down, in place:
//   F_g <- max((max(F_g,0)/dt + S_hi/dg * F_{g+1}) / max(denom, eps), 0)
// with the per-group S_hi/dg and max(denom, eps) precomputed in double in the
// reference's operation order.  The IDD of the new state (Eq. 24 with psi^2 = 0,
// integratedDepthDoseLiteKernel, bfpm_solver.cu:523-591) is accumulated on the
// way as per-block partials; the psi^2 column is 0.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128) lite_energy_kernel(T* __restrict__ F, const double* __restrict__ lc, double dt,
                                                          int Ng, long long lanes, const double* __restrict__ dc,
                                                          int NA, int Ny, int Nz, int trap, double* partials) {
    constexpr int D = 8;  // groups prefetched ahead of use
    const long long lane = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool ok = lane < lanes;
    T ring[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const int e = Ng - 1 - k;
        ring[k] = (ok && e >= 0) ? F[e * lanes + lane] : T(0);
    }
    double w = 1.0;
    if (trap && ok) {
        const int pos = static_cast<int>(lane / NA), iy = pos % (Ny + 1), iz = pos / (Ny + 1);
        if (iy == 0 || iy == Ny) w *= 0.5;
        if (iz == 0 || iz == Nz) w *= 0.5;
    }
    double next = 0.0, acc = 0.0;
    for (int base = Ng - 1; base >= 0; base -= D)
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const int ek = base - k;
        if (ek < 0) break;
        const double Fg = fmax(static_cast<double>(ring[k]), 0.0);
        const int ep = ek - D;
        if (ep >= 0 && ok) ring[k] = F[ep * lanes + lane];
        const double v = fmax((Fg / dt + __ldg(lc + 2 * ek) * next) / __ldg(lc + 2 * ek + 1), 0.0);
        const T vs = static_cast<T>(v);
        if (ok) {
            F[ek * lanes + lane] = vs;
            acc += w * __ldg(dc + 2 * ek) * static_cast<double>(vs);
        }
        next = static_cast<double>(vs);
    }
    __shared__ double red[4];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    const int wi = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[wi] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int i = 0; i < static_cast<int>(blockDim.x >> 5); ++i) a += red[i];
        partials[2 * blockIdx.x] = a;
        partials[2 * blockIdx.x + 1] = 0.0;
    }
}

int lite_energy_grid(long long lanes) { return static_cast<int>((lanes + 127) / 128); }

template <typename T>
cudaError_t launch_lite_energy(T* F, const double* lc, double dt, int Ng, long long lanes, const double* dc, int NA,
                               int Ny, int Nz, int trap, double* partials, cudaStream_t s) {
    lite_energy_kernel<T><<<lite_energy_grid(lanes), 128, 0, s>>>(F, lc, dt, Ng, lanes, dc, NA, Ny, Nz, trap, partials);
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
//
// x with its sign flipped where s has its sign bit set: sign(s) * x for
// s != 0, done on the bits (one logic op instead of a compare and a multiply).
__device__ __forceinline__ float flip_by_sign(float x, float s) {
    return __int_as_float(__float_as_int(x) ^ (__float_as_int(s) & static_cast<int>(0x80000000u)));
}
__device__ __forceinline__ double flip_by_sign(double x, double s) {
    return __longlong_as_double(__double_as_longlong(x) ^
                                (__double_as_longlong(s) & static_cast<long long>(0x8000000000000000ull)));
}

// superbee_diff(back, fwd) takes the two differences of the triple around a
// face.  b = sg * back and the slope sg * m are the sign flips above
// (fwd = -0 flips where sg = +1 would not, but then |fwd| < eps and the
// slope is 0 either way).
template <typename T>
__device__ __forceinline__ T superbee_diff(T back, T fwd) {
    const T af = fabs(fwd), b = flip_by_sign(back, fwd);
    const T m = max(T(0), max(min(b + b, af), min(b, af + af)));
    return af < static_cast<T>(kEpsilon) ? T(0) : flip_by_sign(m, fwd);
}

template <typename T>
__device__ __forceinline__ T superbee(T l, T c, T r) {
    return superbee_diff(c - l, r - c);
}

// A rectangle of positions [y0, y1) x [z0, z1) of one energy plane, staged in
// shared memory with AC angles per position (angle fastest).
struct Rect {
    int y0, y1, z0, z1;
    __device__ int w() const { return y1 - y0; }
    __device__ int h() const { return z1 - z0; }
    __device__ int n() const { return (y1 - y0) * (z1 - z0); }
    __device__ int at(int gy, int gz) const { return (gz - z0) * (y1 - y0) + (gy - y0); }
    __device__ Rect grow(int m, int Ny1, int Nz1) const {
        return Rect{max(0, y0 - m), min(Ny1, y1 + m), max(0, z0 - m), min(Nz1, z1 + m)};
    }
};

// One-dimensional upwind MUSCL flux divergence along a line of a field X
// (spatial_flux_divergence_value, spatial_transport.cu:31-102, one axis).
// With h = 0.5 sgn(w) and face values G(j) = X(j) + h * s(j), where s(j) is the
// limited slope of the clamped triple around j, the divergence at i is
// w (G(i) - G(i-1)) for w >= 0 and w (G(i+1) - G(i)) for w < 0.  Evaluating
// G at j = -1 or N+1 on clamped indices gives X(0) or X(N) exactly (the slope
// of a constant triple is 0), which is the reference's boundary flux, so the
// walk needs no special cases.  The line is walked i = i0 .. i1-1 with a
// sliding window: one load and one slope per step.
// ld(j) reads X at a clamped index j in [0, N]; emit(i, div) consumes div(i).
template <typename T, typename Ld, typename Emit>
__device__ __forceinline__ void walk_line(const Ld& ld, const Emit& emit, int i0, int i1, int N, T w, T rd) {
    const T h = w >= T(0) ? T(0.5) : T(-0.5);
    const bool up = w >= T(0);
    auto X = [&](int j) { return ld(min(max(j, 0), N)); };
    // window: x1 = X(i-1), x2 = X(i), x3 = X(i+1), x4 = X(i+2); faces g0 = G(i-1), g1 = G(i)
    T x0 = X(i0 - 2), x1 = X(i0 - 1), x2 = X(i0), x3 = X(i0 + 1);
    T g0 = x1 + h * superbee(x0, x1, x2);
    T g1 = x2 + h * superbee(x1, x2, x3);
    for (int i = i0; i < i1; ++i) {
        const T x4 = X(i + 2);
        const T g2 = x3 + h * superbee(x2, x3, x4);  // G(i+1)
        const T lf = w * (up ? g0 : g1);
        const T rf = w * (up ? g1 : g2);
        emit(i, (rf - lf) * rd);
        g0 = g1;
        g1 = g2;
        x2 = x3;
        x3 = x4;
    }
}

// One block = one energy group, AC consecutive angles, one tile of output
// positions.  Shared memory holds F over the tile plus a 4-cell halo, the
// y-part of a divergence and the predictor (2-cell halo).  Each stage is two
// line walks: threads (row z, angle) walk y and store the y-part; threads
// (column y, angle) walk z, add the z-part and form the predictor (stage 1)
// or the corrector (stage 2).  H = F - dt/2 div F is written over F in place
// (a column's walk never reads behind itself).  Warps run along angles, so
// every shared access is a contiguous row of AC values.
template <typename T, int AC>
__global__ void __launch_bounds__(512) transport_kernel(TransportArgs<T> a, int tiles_y, int tiles_z, int n_chunks) {
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
    const Rect r2 = t.grow(2, Ny1, Nz1), r4 = t.grow(4, Ny1, Nz1);
    T* Fs = reinterpret_cast<T*>(smem_raw);
    T* Ds = Fs + r4.n() * AC;
    T* Ps = Ds + r2.n() * AC;
    const int a0 = chunk * AC;
    const size_t plane = static_cast<size_t>(ek) * Ny1 * Nz1 * NA + a0;
    const T* __restrict__ in = a.in + plane;
    T* __restrict__ out = a.out + plane;
    const T dt = a.dt, hdt = T(0.5) * a.dt, rdy = T(1) / a.dy, rdz = T(1) / a.dz;
    const int q = threadIdx.x % AC, lane0 = threadIdx.x / AC, lstep = blockDim.x / AC;
    const bool qok = a0 + q < NA;
    const int ang = min(a0 + q, NA - 1);
    const T wy = a.omega[2 * ang], wz = a.omega[2 * ang + 1];

    for (int e = threadIdx.x; e < r4.n() * AC; e += blockDim.x) {
        const int aa = e % AC, p = e / AC;
        const int gz = r4.z0 + p / r4.w(), gy = r4.y0 + p % r4.w();
        Fs[e] = (a0 + aa < NA) ? in[(static_cast<size_t>(gz) * Ny1 + gy) * NA + aa] : T(0);
    }
    __syncthreads();
    // stage 1, y-part of div F over r2
    for (int gz = r2.z0 + lane0; gz < r2.z1; gz += lstep)
        walk_line<T>([&](int y) { return Fs[r4.at(y, gz) * AC + q]; },
                     [&](int y, T d) { Ds[r2.at(y, gz) * AC + q] = d; }, r2.y0, r2.y1, Ny, wy, rdy);
    __syncthreads();
    // stage 1, z-part; predictor over r2, H over the tile (in place of F)
    for (int gy = r2.y0 + lane0; gy < r2.y1; gy += lstep) {
        const bool col_in_t = gy >= t.y0 && gy < t.y1;
        walk_line<T>([&](int z) { return Fs[r4.at(gy, z) * AC + q]; },
                     [&](int z, T dz) {
                         const int ip = r2.at(gy, z) * AC + q, iF = r4.at(gy, z) * AC + q;
                         const T d = Ds[ip] + dz;
                         const T f = Fs[iF];
                         const T v = f - dt * d;
                         Ps[ip] = a.preserve_sign ? v : max(v, T(0));
                         if (col_in_t && z >= t.z0 && z < t.z1) Fs[iF] = f - hdt * d;
                     },
                     r2.z0, r2.z1, Nz, wz, rdz);
    }
    __syncthreads();
    // stage 2, y-part of div P over the tile
    for (int gz = t.z0 + lane0; gz < t.z1; gz += lstep)
        walk_line<T>([&](int y) { return Ps[r2.at(y, gz) * AC + q]; },
                     [&](int y, T d) { Ds[r2.at(y, gz) * AC + q] = d; }, t.y0, t.y1, Ny, wy, rdy);
    __syncthreads();
    // stage 2, z-part and corrector
    for (int gy = t.y0 + lane0; gy < t.y1; gy += lstep)
        walk_line<T>([&](int z) { return Ps[r2.at(gy, z) * AC + q]; },
                     [&](int z, T dz) {
                         const T d = Ds[r2.at(gy, z) * AC + q] + dz;
                         const T v = Fs[r4.at(gy, z) * AC + q] - hdt * d;
                         if (qok) out[(static_cast<size_t>(z) * Ny1 + gy) * NA + q] = a.preserve_sign ? v : max(v, T(0));
                     },
                     t.z0, t.z1, Nz, wz, rdz);
}

// Shared memory of one transport block for a tile of ty x tz positions.
size_t transport_smem(int Ny1, int Nz1, int ty, int tz, int ac, size_t elem) {
    auto n = [&](int h) {
        return static_cast<size_t>(std::min(Ny1, ty + 2 * h)) * std::min(Nz1, tz + 2 * h);
    };
    return (n(4) + 2 * n(2)) * ac * elem;
}

template <typename T, int AC>
static cudaError_t launch_transport_ac(const TransportArgs<T>& a, cudaStream_t s) {
    const int Ny1 = a.Ny + 1, Nz1 = a.Nz + 1;
    const int tiles_y = (Ny1 + a.tile_y - 1) / a.tile_y, tiles_z = (Nz1 + a.tile_z - 1) / a.tile_z;
    const int n_chunks = (a.NA + AC - 1) / AC;
    const size_t smem = transport_smem(Ny1, Nz1, a.tile_y, a.tile_z, AC, sizeof(T));
    auto kern = transport_kernel<T, AC>;
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
    if (e != cudaSuccess) return e;
    const long long blocks = static_cast<long long>(a.Ng) * n_chunks * tiles_y * tiles_z;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    // one thread per (line, angle) of the longest stage-1 walk set, in whole warps, at most 512
    const int lines = std::max(std::min(Ny1, a.tile_y + 4), std::min(Nz1, a.tile_z + 4));
    const int threads = std::min(512, std::max(32, (lines * AC + 31) / 32 * 32));
    kern<<<static_cast<unsigned>(blocks), (threads / AC) * AC, smem, s>>>(a, tiles_y, tiles_z, n_chunks);
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
// Whole-plane transport for square planes of compile-time size.
//
// One block = one energy group and AC consecutive angles of an NP x NP plane
// (NP = Ny+1 = Nz+1), staged whole in shared memory with rows padded to an
// odd length (conflict-free row walks).  Every line walk is unrolled at
// compile time, so shared-memory offsets are immediates and the clamped ends
// fold away.  The numerics are those of walk_line: with face values
// G(-1) = G(0) = X(0), G(N) = G(N+1) = X(N) (the slope of a clamped triple at
// either end is 0) and D(j) = w (G(j) - G(j-1)) / h, the divergence at cell i
// is D(i) for w >= 0 and D(i+1) for w < 0; a thread computes each D(j) once
// and writes it to cell j - s, s = (w < 0), and the cell that receives
// D(0) = 0 or D(N+1) = 0 is handled after the walk.  Two shared planes: F
// (then H = F - dt/2 div F, then H - dt/2 d_y P) and the y-part of div F
// (then the predictor P).
// ---------------------------------------------------------------------------
// Walks X[0], X[S], ..., X[N*S] and calls emit(j, D(j), X(j), X(j-1)) for
// j = 1..N.
template <typename T, int N, int S, typename Emit>
__device__ __forceinline__ void walk_plane_line(const T* X, T wr, T h, const Emit& emit) {
    T xp = X[0];  // X(j-1)
    T xn = X[S];  // X(j)
    T fwd = xn - xp;
    T gp = xp;    // G(0)
#pragma unroll
    for (int j = 1; j < N; ++j) {
        const T xnn = X[(j + 1) * S];
        const T back = fwd;
        fwd = xnn - xn;
        const T g = xn + h * superbee_diff(back, fwd);
        emit(j, wr * (g - gp), xn, xp);
        gp = g;
        xp = xn;
        xn = xnn;
    }
    emit(N, wr * (xn - gp), xn, xp);  // G(N) = X(N)
}

// The same walk with its loads issued kPrefetch steps ahead of their use, in
// program order before the stores of the steps in between (a walk only
// stores to cells it has already read, so nothing is read stale), and with a
// second line Y (stride SY) loaded alongside and handed to emit as
// emit(j, D(j), X(j), X(j-1), Y[j*SY]).
constexpr int kPrefetch = 4;
template <typename T, int N, int S, int SY, bool HY, typename Emit>
__device__ __forceinline__ void walk_plane_line_pf(const T* X, const T* Y, T wr, T h, const Emit& emit) {
    T x[N + 1], y[N + 1];
#pragma unroll
    for (int k = 0; k <= N && k <= kPrefetch + 1; ++k) x[k] = X[k * S];
    if constexpr (HY) {
#pragma unroll
        for (int k = 1; k <= N && k <= kPrefetch; ++k) y[k] = Y[k * SY];
    }
    T fwd = x[1] - x[0];
    T gp = x[0];
#pragma unroll
    for (int j = 1; j < N; ++j) {
        if (j + 1 + kPrefetch <= N) x[j + 1 + kPrefetch] = X[(j + 1 + kPrefetch) * S];
        if constexpr (HY) {
            if (j + kPrefetch <= N) y[j + kPrefetch] = Y[(j + kPrefetch) * SY];
        }
        const T back = fwd;
        fwd = x[j + 1] - x[j];
        const T g = x[j] + h * superbee_diff(back, fwd);
        emit(j, wr * (g - gp), x[j], x[j - 1], HY ? y[j] : T(0));
        gp = g;
    }
    emit(N, wr * (x[N] - gp), x[N], x[N - 1], HY ? y[N] : T(0));  // G(N) = X(N)
}

template <typename T, int NP, int AC>
__global__ void __launch_bounds__((NP * AC + 31) / 32 * 32) transport_plane_kernel(TransportArgs<T> a, int n_chunks) {
    constexpr int N = NP - 1, RP = NP | 1, RS = RP * AC, PL = NP * RS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* Fs = reinterpret_cast<T*>(smem_raw);
    T* Ps = Fs + PL;
    const int chunk = blockIdx.x % n_chunks, ek = blockIdx.x / n_chunks;
    const int NA = a.NA, a0 = chunk * AC;
    const size_t plane = static_cast<size_t>(ek) * NP * NP * NA + a0;
    const T* __restrict__ in = a.in + plane;
    T* __restrict__ out = a.out + plane;
    const int q = threadIdx.x % AC, line = threadIdx.x / AC;
    const bool qok = a0 + q < NA;
    const int ang = min(a0 + q, NA - 1);
    const T wy = a.omega[2 * ang], wz = a.omega[2 * ang + 1];
    const T wry = wy / a.dy, wrz = wz / a.dz;
    const bool dny = wy < T(0), dnz = wz < T(0);
    const T hy = dny ? T(-0.5) : T(0.5), hz = dnz ? T(-0.5) : T(0.5);
    const int sy = dny ? 1 : 0, sz = dnz ? 1 : 0;
    const T dt = a.dt, hdt = T(0.5) * a.dt;
    const T lo = a.preserve_sign ? -INFINITY : T(0);

    constexpr int NT = (NP * AC + 31) / 32 * 32;  // == blockDim.x
    if (AC % Vec16<T>::W == 0 && NA % Vec16<T>::W == 0) {
        // 16-byte pieces by cp.async, all in flight at once (a0 and NA are
        // multiples of the vector width, so a piece is wholly inside or wholly past NA)
        constexpr int W = Vec16<T>::W, NV = NP * NP * AC / W;
#pragma unroll 4
        for (int v = threadIdx.x; v < NV; v += NT) {
            const int e = v * W, aa = e % AC, p = e / AC;
            const int z = p / NP, y = p - z * NP;
            const bool ok = a0 + aa < NA;
            cp_async16(Fs + z * RS + y * AC + aa, ok ? in + static_cast<size_t>(p) * NA + aa : in, ok);
        }
        cp_async_wait_all();
    } else {
#pragma unroll 4
        for (int e = threadIdx.x; e < NP * NP * AC; e += NT) {
            const int aa = e % AC, p = e / AC;
            const int z = p / NP, y = p - z * NP;
            Fs[z * RS + y * AC + aa] = (a0 + aa < NA) ? in[static_cast<size_t>(p) * NA + aa] : T(0);
        }
    }
    __syncthreads();
    const bool act = line < NP;
    // stage 1, y-part of div F (rows z = line) into Ps
    if (act) {
        const T* X = Fs + line * RS + q;
        T* D = Ps + line * RS + q - sy * AC;
        walk_plane_line_pf<T, N, AC, 0, false>(X, nullptr, wry, hy, [&](int j, T d, T, T, T) { D[j * AC] = d; });
        Ps[line * RS + q + sy * N * AC] = T(0);
    }
    __syncthreads();
    // stage 1, z-part (columns y = line): predictor into Ps, H over F
    if (act) {
        T* Xc = Fs + line * AC + q;
        T* Pc = Ps + line * AC + q;
        T* Xe = Xc - sz * RS;
        T* Pe = Pc - sz * RS;
        walk_plane_line_pf<T, N, RS, RS, true>(Xc, Pe, wrz, hz, [&](int j, T dz, T xj, T xjm1, T pj) {
            const T f = dnz ? xjm1 : xj;
            const T d = pj + dz;
            Pe[j * RS] = max(f - dt * d, lo);
            Xe[j * RS] = f - hdt * d;
        });
        const int cb = sz * N * RS;  // the cell whose z-part is 0
        const T f = Xc[cb], d = Pc[cb];
        Pc[cb] = max(f - dt * d, lo);
        Xc[cb] = f - hdt * d;
    }
    __syncthreads();
    // stage 2, y-part of div P (rows): H - dt/2 d_y P over F
    if (act) {
        const T* X = Ps + line * RS + q;
        T* Fe = Fs + line * RS + q - sy * AC;
        walk_plane_line_pf<T, N, AC, AC, true>(X, Fe, wry, hy,
                                               [&](int j, T d, T, T, T fj) { Fe[j * AC] = fj - hdt * d; });
    }
    __syncthreads();
    // stage 2, z-part (columns) and the corrector, to global
    if (act) {
        const T* X = Ps + line * AC + q;
        const T* Fc = Fs + line * AC + q;
        const T* Fe = Fc - sz * RS;
        T* o = out + static_cast<size_t>(line) * NA + q;
        const size_t zs = static_cast<size_t>(NP) * NA;
        T* oe = o - sz * zs;
        walk_plane_line_pf<T, N, RS, RS, true>(X, Fe, wrz, hz, [&](int j, T d, T, T, T fj) {
            const T v = max(fj - hdt * d, lo);
            if (qok) oe[j * zs] = v;
        });
        const int cb = sz * N;
        if (qok) o[cb * zs] = max(Fc[cb * RS], lo);
    }
}

// ---------------------------------------------------------------------------
// The same whole-plane kernel with two angles per thread (float state; the
// two share the signs of omega_y and omega_z, checked on the host).  Sums,
// products and shared-memory moves work on fp32x2 pairs; the limiter's
// compares stay per angle.  Each operation is the scalar kernel's, so the
// results agree with it value for value (up to the sign of zeros).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 sub2(float2 x, float2 y) {  // x - y, one rounding
    return __ffma2_rn(y, make_float2(-1.f, -1.f), x);
}

// sign(fwd) where |fwd| >= eps, +-0 below: set gives 1.0f / 0.0f, the sign bit of fwd is or-ed in.
__device__ __forceinline__ float sign_or_zero(float fwd) {
    float st;
    asm("set.ge.f32.f32 %0, %1, %2;" : "=f"(st) : "f"(fabsf(fwd)), "f"(static_cast<float>(kEpsilon)));
    return __int_as_float(__float_as_int(st) | (__float_as_int(fwd) & static_cast<int>(0x80000000u)));
}

// min(|x|, |y|) carrying the sign bit sign(x) xor sign(y): negative exactly
// when x and y have opposite signs.
__device__ __forceinline__ float min_xorsign_abs(float x, float y) {
    float d;
    asm("min.xorsign.abs.f32 %0, %1, %2;" : "=f"(d) : "f"(x), "f"(y));
    return d;
}

// max(x, y, z) in one instruction (sm_100).
__device__ __forceinline__ float max3f(float x, float y, float z) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(x), "f"(y), "f"(z));
    return d;
}

// superbee_diff for a pair, from the two differences around the face and
// their doubles (2 back is the previous face's 2 fwd, so each double is
// formed once).  With b = sgn(fwd) back: min_xorsign_abs(2 back, fwd) is
// min(2b, |fwd|) when back and fwd share a sign and negative otherwise (so is
// min(2b, |fwd|) then, b being negative), and likewise min(back, 2 fwd) ~
// min(b, 2|fwd|); m = max(0, both) is the scalar form's m value for value.
// The slope is sign_or_zero(fwd) m: sgn(fwd) m, and 0 below eps.
__device__ __forceinline__ float2 superbee_diff2(float2 back, float2 back2, float2 fwd, float2 fwd2) {
    float2 m;
    m.x = max3f(0.f, min_xorsign_abs(back2.x, fwd.x), min_xorsign_abs(back.x, fwd2.x));
    m.y = max3f(0.f, min_xorsign_abs(back2.y, fwd.y), min_xorsign_abs(back.y, fwd2.y));
    return __fmul2_rn(m, make_float2(sign_or_zero(fwd.x), sign_or_zero(fwd.y)));
}

template <int N, int S, int SY, bool HY, typename Emit>
__device__ __forceinline__ void walk_plane_line2(const float2* X, const float2* Y, float2 wr, float2 h,
                                                 const Emit& emit) {
    float2 x[N + 1], y[N + 1];
#pragma unroll
    for (int k = 0; k <= N && k <= kPrefetch + 1; ++k) x[k] = X[k * S];
    if constexpr (HY) {
#pragma unroll
        for (int k = 1; k <= N && k <= kPrefetch; ++k) y[k] = Y[k * SY];
    }
    float2 fwd = sub2(x[1], x[0]);
    float2 fwd2 = __fadd2_rn(fwd, fwd);
    float2 gp = x[0];
#pragma unroll
    for (int j = 1; j < N; ++j) {
        if (j + 1 + kPrefetch <= N) x[j + 1 + kPrefetch] = X[(j + 1 + kPrefetch) * S];
        if constexpr (HY) {
            if (j + kPrefetch <= N) y[j + kPrefetch] = Y[(j + kPrefetch) * SY];
        }
        const float2 back = fwd, back2 = fwd2;
        fwd = sub2(x[j + 1], x[j]);
        fwd2 = __fadd2_rn(fwd, fwd);
        const float2 g = __ffma2_rn(h, superbee_diff2(back, back2, fwd, fwd2), x[j]);
        emit(j, __fmul2_rn(wr, sub2(g, gp)), x[j], x[j - 1], HY ? y[j] : make_float2(0.f, 0.f));
        gp = g;
    }
    emit(N, __fmul2_rn(wr, sub2(x[N], gp)), x[N], x[N - 1], HY ? y[N] : make_float2(0.f, 0.f));
}

__device__ __forceinline__ float2 max_lo2(float2 v, float lo) { return make_float2(fmaxf(v.x, lo), fmaxf(v.y, lo)); }



template <int NP, int AC>
__device__ __forceinline__ void transport_plane_f2_body(const TransportArgs<float>& a, int n_chunks, int bid) {
    constexpr int N = NP - 1, RP = NP | 1, A2 = AC / 2, RS = RP * A2, PL = NP * RS;  // in float2
    constexpr int NT = (NP * A2 + 31) / 32 * 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* Fs = reinterpret_cast<float2*>(smem_raw);
    float2* Ps = Fs + PL;
    const int chunk = bid % n_chunks, ek = bid / n_chunks;
    const int NA = a.NA, a0 = chunk * AC;
    const size_t plane = static_cast<size_t>(ek) * NP * NP * NA + a0;
    const float* __restrict__ in = a.in + plane;
    float* __restrict__ out = a.out + plane;
    const int q = threadIdx.x % A2, line = threadIdx.x / A2;  // angles a0 + 2q, a0 + 2q + 1
    const bool ok0 = a0 + 2 * q < NA, ok1 = a0 + 2 * q + 1 < NA;
    const int g0 = min(a0 + 2 * q, NA - 1), g1 = min(a0 + 2 * q + 1, NA - 1);
    const float wy0 = a.omega[2 * g0], wz0 = a.omega[2 * g0 + 1];
    const float wy1 = a.omega[2 * g1], wz1 = a.omega[2 * g1 + 1];
    const float2 wry = make_float2(wy0 / a.dy, wy1 / a.dy), wrz = make_float2(wz0 / a.dz, wz1 / a.dz);
    const bool dny = wy0 < 0.f, dnz = wz0 < 0.f;
    const float2 hy = dny ? make_float2(-0.5f, -0.5f) : make_float2(0.5f, 0.5f);
    const float2 hz = dnz ? make_float2(-0.5f, -0.5f) : make_float2(0.5f, 0.5f);
    const int sy = dny ? 1 : 0, sz = dnz ? 1 : 0;
    const float2 ndt = make_float2(-a.dt, -a.dt), nhdt = make_float2(-0.5f * a.dt, -0.5f * a.dt);
    const float lo = a.preserve_sign ? -INFINITY : 0.f;

    float* Fsf = reinterpret_cast<float*>(Fs);
    if (AC % 4 == 0 && NA % 4 == 0) {
        // every 16-byte piece of the plane in flight at once
        constexpr int NV = NP * NP * AC / 4;
#pragma unroll 4
        for (int v = threadIdx.x; v < NV; v += NT) {
            const int e = v * 4, aa = e % AC, p = e / AC;
            const int z = p / NP, y = p - z * NP;
            const bool ok = a0 + aa < NA;
            cp_async16(Fsf + 2 * (z * RS + y * A2) + aa, ok ? in + static_cast<size_t>(p) * NA + aa : in, ok);
        }
        cp_async_wait_all();
    } else {
#pragma unroll 4
        for (int e = threadIdx.x; e < NP * NP * AC; e += NT) {
            const int aa = e % AC, p = e / AC;
            const int z = p / NP, y = p - z * NP;
            Fsf[2 * (z * RS + y * A2) + aa] = (a0 + aa < NA) ? in[static_cast<size_t>(p) * NA + aa] : 0.f;
        }
    }
    __syncthreads();
    const bool act = line < NP;
    // stage 1, y-part of div F (rows z = line) into Ps
    if (act) {
        const float2* X = Fs + line * RS + q;
        float2* D = Ps + line * RS + q - sy * A2;
        walk_plane_line2<N, A2, 0, false>(X, nullptr, wry, hy, [&](int j, float2 d, float2, float2, float2) {
            D[j * A2] = d;
        });
        Ps[line * RS + q + sy * N * A2] = make_float2(0.f, 0.f);
    }
    __syncthreads();
    // stage 1, z-part (columns y = line): predictor into Ps, H over F
    if (act) {
        float2* Xc = Fs + line * A2 + q;
        float2* Pc = Ps + line * A2 + q;
        float2* Xe = Xc - sz * RS;
        float2* Pe = Pc - sz * RS;
        walk_plane_line2<N, RS, RS, true>(Xc, Pe, wrz, hz, [&](int j, float2 dz, float2 xj, float2 xjm1, float2 pj) {
            const float2 f = dnz ? xjm1 : xj;
            const float2 d = __fadd2_rn(pj, dz);
            Pe[j * RS] = max_lo2(__ffma2_rn(ndt, d, f), lo);
            Xe[j * RS] = __ffma2_rn(nhdt, d, f);
        });
        const int cb = sz * N * RS;
        const float2 f = Xc[cb], d = Pc[cb];
        Pc[cb] = max_lo2(__ffma2_rn(ndt, d, f), lo);
        Xc[cb] = __ffma2_rn(nhdt, d, f);
    }
    __syncthreads();
    // stage 2, y-part of div P (rows): H - dt/2 d_y P over F
    if (act) {
        const float2* X = Ps + line * RS + q;
        float2* Fe = Fs + line * RS + q - sy * A2;
        walk_plane_line2<N, A2, A2, true>(X, Fe, wry, hy, [&](int j, float2 d, float2, float2, float2 fj) {
            Fe[j * A2] = __ffma2_rn(nhdt, d, fj);
        });
    }
    __syncthreads();
    // stage 2, z-part (columns) and the corrector, to global
    if (act) {
        const float2* X = Ps + line * A2 + q;
        const float2* Fc = Fs + line * A2 + q;
        const float2* Fe = Fc - sz * RS;
        float* o = out + static_cast<size_t>(line) * NA + 2 * q;
        const size_t zs = static_cast<size_t>(NP) * NA;
        float* oe = o - sz * zs;
        auto put = [&](float* dst, float2 v) {
            if (ok1) *reinterpret_cast<float2*>(dst) = v;
            else if (ok0) *dst = v.x;
        };
        walk_plane_line2<N, RS, RS, true>(X, Fe, wrz, hz, [&](int j, float2 d, float2, float2, float2 fj) {
            put(oe + j * zs, max_lo2(__ffma2_rn(nhdt, d, fj), lo));
        });
        const int cb = sz * N;
        put(o + cb * zs, max_lo2(Fc[cb * RS], lo));
    }
}

template <int NP, int AC>
__global__ void __launch_bounds__((NP * AC / 2 + 31) / 32 * 32) transport_plane_f2_kernel(TransportArgs<float> a,
                                                                                           int n_chunks) {
    transport_plane_f2_body<NP, AC>(a, n_chunks, blockIdx.x);
}

template <int NP, int AC>
__global__ void __launch_bounds__((NP * AC / 2 + 31) / 32 * 32)
    transport_plane_f2_slots_kernel(const TransportArgs<float>* __restrict__ args, const int* __restrict__ begin,
                                    int nslots, int n_chunks) {
    const int s = find_slot(begin, nslots, blockIdx.x);
    transport_plane_f2_body<NP, AC>(args[s], n_chunks, blockIdx.x - __ldg(begin + s));
}

// ---------------------------------------------------------------------------
// Planes too large for one block (float state, paired angles): a cluster of
// CL CTAs holds one (group, 2*A2-angle chunk) plane, CTA r the z rows
// [r NP / CL, (r+1) NP / CL) of both shared planes (F, then H; the y-part of
// div F, then the predictor P).  No cell is computed twice.  Row walks are
// local: a row is cut into YS segments, each walked by its own thread from
// its cells plus 2 either side.  Column walks take their band plus 2 rows
// either side: in stage 1 those rows come from the input in HBM, in stage 2
// from the neighbouring CTAs' predictor rows (distributed shared memory),
// behind a cluster barrier whose arrive follows each CTA's stage 1 and whose
// wait precedes its stage 2.  Cells beyond the plane repeat the edge value
// (the reference's clamped indices), which also yields D = 0 at the boundary
// face.  Per cell the arithmetic is the whole-plane kernel's.
// ---------------------------------------------------------------------------
template <int NP, int CL, int A2>
struct ClusterPlane {
    static constexpr int N = NP - 1;
    static constexpr int BZ = (NP + CL - 1) / CL;         // rows of the largest band
    static constexpr int YS = (NP + BZ - 1) / BZ;         // row segments
    static constexpr int SL = (NP + YS - 1) / YS;         // cells of the longest segment
    static constexpr int YT = (BZ * A2 + 31) / 32 * 32;   // threads per row segment
    static constexpr int NT = (NP * A2 > YS * YT ? (NP * A2 + 31) / 32 * 32 : YS * YT);
    static constexpr int RS = NP * A2;                    // row stride (float2)
    static constexpr size_t smem = 2ull * BZ * RS * sizeof(float2);
};

// One line of faces: D(j) = wr (G(j) - G(j-1)), G(j) = x_j + h sb(x_j - x_{j-1},
// x_{j+1} - x_j), over values x_k = get(k), k = 0 .. L-1, standing for
// X(first - 2) .. X(first + L - 3); emit(i, d, X(first + i - 1), X(first + i))
// for face first + i, i = 0 .. L-4.  get(k) is called kPrefetch steps ahead of
// its use, in program order before the emits in between (which only store to
// cells already read).
template <int L, typename Get, typename Emit>
__device__ __forceinline__ void walk_get2(const Get& get, float2 wr, float2 h, const Emit& emit) {
    float2 x[L];
#pragma unroll
    for (int k = 0; k < L && k < kPrefetch + 3; ++k) x[k] = get(k);
    float2 back = sub2(x[1], x[0]);
    float2 fwd = sub2(x[2], x[1]);
    float2 back2 = __fadd2_rn(back, back), fwd2 = __fadd2_rn(fwd, fwd);
    float2 gp = __ffma2_rn(h, superbee_diff2(back, back2, fwd, fwd2), x[1]);  // G(first - 1)
#pragma unroll
    for (int i = 0; i + 4 <= L; ++i) {
        if (i + 3 + kPrefetch < L) x[i + 3 + kPrefetch] = get(i + 3 + kPrefetch);
        back = fwd;
        back2 = fwd2;
        fwd = sub2(x[i + 3], x[i + 2]);
        fwd2 = __fadd2_rn(fwd, fwd);
        const float2 g = __ffma2_rn(h, superbee_diff2(back, back2, fwd, fwd2), x[i + 2]);
        emit(i, __fmul2_rn(wr, sub2(g, gp)), x[i + 1], x[i + 2]);
        gp = g;
    }
}

// Row segment [c0, c1) of a row at X (stride A2), c1 - c0 <= SL: faces
// c0 .. c0 + SL (those past c1 are walked on clamped loads and not emitted),
// cell = face - s.  One code path for every segment of a row (small code).
template <int N, int SL, int A2, typename Emit>
__device__ __forceinline__ void walk_row_segment(const float2* X, int c0, int c1, float2 wr, float2 h, int s,
                                                 const Emit& emit) {
    walk_get2<SL + 4>([&](int k) { return X[min(max(c0 - 2 + k, 0), N) * A2]; }, wr, h,
                      [&](int i, float2 d, float2, float2) {
                          const int cell = c0 + i - s;
                          if (cell >= c0 && cell < c1) emit(cell, d);
                      });
}

// Column over a band of B rows (B = BZ or BZ - 1) at Xb (stride RS), with 2
// rows below and 3 above in registers: faces z0 .. z0 + BZ, cell (band row) =
// face - z0 - s, emitted for cells < B; emit gets the X value of the cell as
// its third argument.  One code path for both band heights.
template <int BZ, int RS, typename Emit>
__device__ __forceinline__ void walk_band_column(const float2* Xb, int B, const float2 (&below)[2],
                                                 const float2 (&above)[3], float2 wr, float2 h, int s,
                                                 const Emit& emit) {
    const bool full = B == BZ;
    walk_get2<BZ + 4>(
        [&](int k) {
            if (k < 2) return below[k];
            if (k < BZ + 1) return Xb[(k - 2) * RS];
            if (k == BZ + 1) return full ? Xb[(BZ - 1) * RS] : above[0];
            return full ? above[k - BZ - 2] : above[k - BZ - 1];
        },
        wr, h,
        [&](int i, float2 d, float2 xm, float2 x0) {
            const int cell = i - s;
            if (cell >= 0 && cell < B) emit(cell, d, s ? xm : x0);
        });
}

template <int NP, int CL, int A2>
__device__ __forceinline__ void transport_cluster_body(const TransportArgs<float>& a, int n_chunks, int bid) {
    using S = ClusterPlane<NP, CL, A2>;
    constexpr int N = S::N, BZ = S::BZ, RS = S::RS, AC = 2 * A2;
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* Fs = reinterpret_cast<float2*>(smem_raw);
    float2* Ps = Fs + BZ * RS;
    const int rank = static_cast<int>(cluster.block_rank());
    const int plane_id = bid / CL;
    const int chunk = plane_id % n_chunks, ek = plane_id / n_chunks;
    const int z0 = rank * NP / CL, z1 = (rank + 1) * NP / CL, B = z1 - z0;
    const int NA = a.NA, a0 = chunk * AC;
    const size_t zs = static_cast<size_t>(NP) * NA;  // one z row in the state
    const float* in = a.in + static_cast<size_t>(ek) * NP * zs + a0;
    float* out = a.out + static_cast<size_t>(ek) * NP * zs + a0;
    const int tid = threadIdx.x;

    // column items: (column cy, pair cq); row items: (segment, band row rz, pair rq)
    const int cq = tid % A2, cy = tid / A2;
    const int seg = tid / S::YT, rr = tid % S::YT, rq = rr % A2, rz = rr / A2;
    auto pair_setup = [&](int q, float2& wry, float2& wrz, float2& hy, float2& hz, int& sy, int& sz, bool& ok0,
                          bool& ok1) {
        ok0 = a0 + 2 * q < NA;
        ok1 = a0 + 2 * q + 1 < NA;
        const int g0 = min(a0 + 2 * q, NA - 1), g1 = min(a0 + 2 * q + 1, NA - 1);
        const float wy0 = a.omega[2 * g0], wz0 = a.omega[2 * g0 + 1];
        const float wy1 = a.omega[2 * g1], wz1 = a.omega[2 * g1 + 1];
        wry = make_float2(wy0 / a.dy, wy1 / a.dy);
        wrz = make_float2(wz0 / a.dz, wz1 / a.dz);
        hy = wy0 < 0.f ? make_float2(-0.5f, -0.5f) : make_float2(0.5f, 0.5f);
        hz = wz0 < 0.f ? make_float2(-0.5f, -0.5f) : make_float2(0.5f, 0.5f);
        sy = wy0 < 0.f ? 1 : 0;
        sz = wz0 < 0.f ? 1 : 0;
    };
    const float2 ndt = make_float2(-a.dt, -a.dt), nhdt = make_float2(-0.5f * a.dt, -0.5f * a.dt);
    const float lo = a.preserve_sign ? -INFINITY : 0.f;
    const bool col_item = cy < NP;
    const bool row_item = seg < S::YS && rz < B;

    // stage 0: the band of F; column items also take F 2 rows either side (clamped to the plane)
    float* Fsf = reinterpret_cast<float*>(Fs);
    if (NA % 4 == 0) {  // every 16-byte piece of the band in flight at once
        for (int v = tid; v < B * NP * (AC / 4); v += S::NT) {
            const int hp = v % (AC / 4), p = v / (AC / 4);
            const bool ok = a0 + 4 * hp < NA;
            cp_async16(Fsf + p * (2 * A2) + 4 * hp, ok ? in + static_cast<size_t>(z0 * NP + p) * NA + 4 * hp : in, ok);
        }
    } else {
        for (int v = tid; v < B * NP * A2; v += S::NT) {
            const int q = v % A2, p = v / A2;
            float2 val{};
            if (a0 + 2 * q < NA)
                val = *reinterpret_cast<const float2*>(in + static_cast<size_t>(z0 * NP + p) * NA + 2 * q);
            Fs[p * A2 + q] = val;
        }
    }
    float2 fb[2] = {}, fa[3] = {};
    if (col_item && a0 + 2 * cq < NA) {
        const float* col = in + static_cast<size_t>(cy) * NA + 2 * cq;
        fb[0] = *reinterpret_cast<const float2*>(col + max(z0 - 2, 0) * zs);
        fb[1] = *reinterpret_cast<const float2*>(col + max(z0 - 1, 0) * zs);
#pragma unroll
        for (int k = 0; k < 3; ++k) fa[k] = *reinterpret_cast<const float2*>(col + min(z1 + k, N) * zs);
    }
    if (NA % 4 == 0) cp_async_wait_all();
    __syncthreads();
    // stage 1, y-part of div F (rows) into Ps
    if (row_item) {
        float2 wry, wrz, hy, hz;
        int sy, sz;
        bool ok0, ok1;
        pair_setup(rq, wry, wrz, hy, hz, sy, sz, ok0, ok1);
        float2* D = Ps + rz * RS + rq;
        walk_row_segment<N, S::SL, A2>(Fs + rz * RS + rq, seg * NP / S::YS, (seg + 1) * NP / S::YS, wry, hy, sy,
                                       [&](int cell, float2 d) { D[cell * A2] = d; });
    }
    __syncthreads();
    // stage 1, z-part (columns): predictor into Ps, H over F
    if (col_item) {
        float2 wry, wrz, hy, hz;
        int sy, sz;
        bool ok0, ok1;
        pair_setup(cq, wry, wrz, hy, hz, sy, sz, ok0, ok1);
        float2* Pc = Ps + cy * A2 + cq;
        float2* Xc = Fs + cy * A2 + cq;
        auto emit = [&](int cell, float2 dz, float2 f) {
            const float2 d = __fadd2_rn(Pc[cell * RS], dz);
            Pc[cell * RS] = max_lo2(__ffma2_rn(ndt, d, f), lo);
            Xc[cell * RS] = __ffma2_rn(nhdt, d, f);
        };
        walk_band_column<BZ, RS>(Xc, B, fb, fa, wrz, hz, sz, emit);
    }
    cluster.barrier_arrive();  // this CTA's predictor rows are final
    __syncthreads();
    // stage 2, y-part of div P (rows): H - dt/2 d_y P over F
    if (row_item) {
        float2 wry, wrz, hy, hz;
        int sy, sz;
        bool ok0, ok1;
        pair_setup(rq, wry, wrz, hy, hz, sy, sz, ok0, ok1);
        float2* Fe = Fs + rz * RS + rq;
        walk_row_segment<N, S::SL, A2>(Ps + rz * RS + rq, seg * NP / S::YS, (seg + 1) * NP / S::YS, wry, hy, sy,
                                       [&](int cell, float2 d) { Fe[cell * A2] = __ffma2_rn(nhdt, d, Fe[cell * A2]); });
    }
    __syncthreads();
    cluster.barrier_wait();  // the neighbours' predictor rows are final
    // stage 2, z-part (columns) and the corrector, to HBM
    if (col_item) {
        float2 wry, wrz, hy, hz;
        int sy, sz;
        bool ok0, ok1;
        pair_setup(cq, wry, wrz, hy, hz, sy, sz, ok0, ok1);
        const int off = cy * A2 + cq;
        float2 pb[2], pa[3];
        if (rank > 0) {
            const int Bm = z0 - (rank - 1) * NP / CL;  // rows of the band below
            const float2* rem = cluster.map_shared_rank(Ps, rank - 1);
            pb[0] = rem[(Bm - 2) * RS + off];
            pb[1] = rem[(Bm - 1) * RS + off];
        } else {
            pb[0] = pb[1] = Ps[off];
        }
        if (rank < CL - 1) {
            const float2* rem = cluster.map_shared_rank(Ps, rank + 1);
#pragma unroll
            for (int k = 0; k < 3; ++k) pa[k] = rem[k * RS + off];
        } else {
            pa[0] = pa[1] = pa[2] = Ps[(B - 1) * RS + off];
        }
        const float2* Fc = Fs + off;
        float* o = out + static_cast<size_t>(z0) * zs + static_cast<size_t>(cy) * NA + 2 * cq;
        auto emit = [&](int cell, float2 d, float2) {
            const float2 v = max_lo2(__ffma2_rn(nhdt, d, Fc[cell * RS]), lo);
            float* dst = o + cell * zs;
            if (ok1) *reinterpret_cast<float2*>(dst) = v;
            else if (ok0) *dst = v.x;
        };
        walk_band_column<BZ, RS>(Ps + off, B, pb, pa, wrz, hz, sz, emit);
    }
    cluster.sync();  // no CTA leaves while a neighbour still reads its rows
}

template <int NP, int CL, int A2>
__global__ void __cluster_dims__(CL, 1, 1) __launch_bounds__(ClusterPlane<NP, CL, A2>::NT)
    transport_cluster_kernel(TransportArgs<float> a, int n_chunks) {
    transport_cluster_body<NP, CL, A2>(a, n_chunks, blockIdx.x);
}

// Slot boundaries fall on cluster boundaries (every slot's grid is a
// multiple of CL), so all CTAs of a cluster serve one slot.
template <int NP, int CL, int A2>
__global__ void __cluster_dims__(CL, 1, 1) __launch_bounds__(ClusterPlane<NP, CL, A2>::NT)
    transport_cluster_slots_kernel(const TransportArgs<float>* __restrict__ args, const int* __restrict__ begin,
                                   int nslots, int n_chunks) {
    const int s = find_slot(begin, nslots, blockIdx.x);
    transport_cluster_body<NP, CL, A2>(args[s], n_chunks, blockIdx.x - __ldg(begin + s));
}

// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Row-streaming transport (float state, paired angles), any plane with
// Ny + 1 <= 256: one block per (group, 8-angle chunk) plane walks the z rows
// once.  Two threads per column y, each carrying two of the chunk's four angle
// pairs (fp32x2), keep the column's z-stencil in registers -- the last three
// rows of F, of the predictor P and of H, and the face values G of the z-walk
// -- so the z-parts of both stages are line walks with one limiter per cell
// and no memory traffic.  The y-parts need the whole row: row i of F (staged
// by cp.async a few rows ahead into a ring, one 16-byte piece per thread) and
// row i-2 of P sit in shared memory; each thread forms the y face value at its
// own cells from their two neighbours, publishes it, and takes the
// neighbour's after the barrier.  Iteration i runs stage 1 (predictor P and
// H = F - dt/2 div F) on row i and stage 2 (H - dt/2 div P, clipped) on row
// i-2, whose z-stencil needs P up to row i.  Two barriers per row, no halo
// recomputed, no cluster; the first two and last two rows are peeled out of
// the loop so its body is branch-free.  The per-cell arithmetic and its order
// are those of the whole-plane kernel.  Rows and columns beyond the plane
// repeat the edge value, as the reference's clamped indices do.
// ---------------------------------------------------------------------------
constexpr int kStreamPairs = 4;            // angle pairs per block (8 angles, 32 bytes per position)
constexpr int kStreamRing = 8;             // rows of F in the shared-memory ring
constexpr int kStreamAhead = 5;            // rows copied ahead of the one a row's z-stencil needs
constexpr int kStreamPRows = 4;            // rows of P kept in shared memory (rows i-2 .. i)
constexpr int kStreamPT = 2;               // angle pairs per thread
constexpr int kStreamTPC = kStreamPairs / kStreamPT;  // threads per column
constexpr int kStreamMaxThreads = 256 * kStreamTPC;   // planes up to 256 points wide
// register cap: two blocks per SM at the 81-point plane either way
constexpr int kStreamMaxReg = kStreamPT == 2 ? 168 : 88;

size_t transport_stream_smem(int NPy) {
    const size_t row = static_cast<size_t>(NPy) * kStreamPairs * sizeof(float2);
    const size_t grow = static_cast<size_t>(NPy + 3) * kStreamPairs * sizeof(float2);
    return (kStreamRing + kStreamPRows) * row + 4 * grow;  // face rows of F and P, double-buffered
}

// kStreamTPC threads per column y: thread (y, t) carries angle pairs t,
// t + kStreamTPC, ... of the block's four; threads t < 2 also copy the row's
// 16-byte pieces, one each.  The z-stencil of a pair lives in three-slot register
// rotations indexed by row mod 3; the row loop is unrolled by three so every
// slot index is a compile-time constant and the rotation costs no moves.
struct StreamPair {
    float2 f[3];              // F row r in f[r % 3] (rows i .. i+2 at iteration i)
    float2 p[3], hh[3];       // predictor P and H row r in [r % 3] (rows i-2 .. i)
    float2 gz[3], zf[3], zf2[3];  // z-walk of F: face value of cell c in gz[c % 3]; F(i+2) - F(i+1) and its double in [i % 3]
    float2 pz[3], pf[3], pf2[3];  // z-walk of P: face value of cell c in pz[c % 3]; P(i) - P(i-1) and its double in [i % 3]
    float2 wry, wrz, hy, hz;
    bool dnz;
    int own, offl, offr, ghi, glo;              // shared-memory offsets (float2) in a row / a face row
    bool ok1, ok_half;                          // both angles of the pair inside NA; only the first
};

__device__ __forceinline__ void transport_stream_body(const TransportArgs<float>& a, int n_chunks, int bid) {
    constexpr int A2 = kStreamPairs, AC = 2 * A2, RF = kStreamRing, PD = kStreamAhead, RP = kStreamPRows;
    static_assert((RF & (RF - 1)) == 0 && (RP & (RP - 1)) == 0 && AC == 8, "ring sizes are powers of two");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int Ny = a.Ny, Nz = a.Nz, NPy = Ny + 1, NA = a.NA;
    const int RS = NPy * A2;       // one row, in float2
    const int GS = (NPy + 2) * A2 + A2;  // one face row: faces -1 .. N+1, then a spare row for edge-less threads
    float2* Fr = reinterpret_cast<float2*>(smem_raw);  // [RF][NPy][A2]
    float2* Pr = Fr + RF * RS;                         // [RP][NPy][A2]
    float2* Gb = Pr + RP * RS;                         // [2][F, P][GS]: G of the y-walks, by row parity
    const int chunk = bid % n_chunks, ek = bid / n_chunks, a0 = chunk * AC;
    const size_t zs = static_cast<size_t>(NPy) * NA;  // one z row in the state
    const size_t base = static_cast<size_t>(ek) * (Nz + 1) * zs + a0;
    constexpr int PT = kStreamPT, TPC = kStreamTPC;
    const int tid = threadIdx.x, h = tid % TPC, y = tid / TPC;

    // this thread's 16-byte piece of every row (threads h < 2): position y, angles a0 + 4h .. a0 + 4h + 3
    const bool vec = NA % 4 == 0;
    const bool lcp = h < 2;
    const bool lok = vec && lcp && a0 + 4 * h < NA;
    const float* in0 = a.in;
    const float* lsrc = in0 + base + static_cast<size_t>(y) * NA + 4 * (h & 1);
    float* ldst = reinterpret_cast<float*>(Fr) + y * AC + 4 * (h & 1);
    auto fill = [&](int r) {  // row r of F into slot r % RF; one commit group per call, empty past the plane
        if (r <= Nz) {
            if (vec) {
                if (lcp) cp_async16(ldst + (r & (RF - 1)) * (2 * RS), lok ? lsrc + static_cast<size_t>(r) * zs : in0, lok);
            } else {
                float* row = reinterpret_cast<float*>(Fr + (r & (RF - 1)) * RS);
                const float* src = in0 + base + static_cast<size_t>(r) * zs;
                for (int v = tid; v < NPy * AC; v += blockDim.x) {
                    const int e = v % AC, p = v / AC;
                    row[p * AC + e] = (a0 + e < NA) ? src[static_cast<size_t>(p) * NA + e] : 0.f;
                }
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };

    const float2 ndt = make_float2(-a.dt, -a.dt), nhdt = make_float2(-0.5f * a.dt, -0.5f * a.dt);
    const float lo = a.preserve_sign ? -INFINITY : 0.f;
    // the face beyond the plane (edge threads) or a spare slot (the others): every thread stores one
    const int gedge_row = y == 0 ? 0 : (y == Ny ? (NPy + 1) * A2 : (NPy + 2) * A2);
    StreamPair S[PT];
#pragma unroll
    for (int k = 0; k < PT; ++k) {
        StreamPair& P = S[k];
        const int q = h + TPC * k;
        P.ok1 = a0 + 2 * q + 1 < NA;
        P.ok_half = a0 + 2 * q < NA && !P.ok1;
        const int g0 = min(a0 + 2 * q, NA - 1), g1 = min(a0 + 2 * q + 1, NA - 1);
        const float wy0 = a.omega[2 * g0], wz0 = a.omega[2 * g0 + 1];
        const float wy1 = a.omega[2 * g1], wz1 = a.omega[2 * g1 + 1];
        P.wry = make_float2(wy0 / a.dy, wy1 / a.dy);
        P.wrz = make_float2(wz0 / a.dz, wz1 / a.dz);
        const bool dny = wy0 < 0.f;
        P.dnz = wz0 < 0.f;
        P.hy = dny ? make_float2(-0.5f, -0.5f) : make_float2(0.5f, 0.5f);
        P.hz = P.dnz ? make_float2(-0.5f, -0.5f) : make_float2(0.5f, 0.5f);
        P.own = y * A2 + q;
        P.offl = max(y - 1, 0) * A2 + q;
        P.offr = min(y + 1, Ny) * A2 + q;
        // G index of the two faces of this cell's y-divergence (G is stored one face up)
        P.ghi = P.own + (dny ? 2 * A2 : A2);
        P.glo = P.own + (dny ? A2 : 0);
#pragma unroll
        for (int r = 0; r < 3; ++r) P.p[r] = P.hh[r] = make_float2(0.f, 0.f);
    }
    float* orow = a.out + base + static_cast<size_t>(y) * NA;  // this position's angles a0 .. a0+7, row 0

    auto y_face = [&](float2* G, const float2* row, const StreamPair& P, float2 x) {
        const float2 back = sub2(x, row[P.offl]), fwd = sub2(row[P.offr], x);
        G[P.own + A2] = __ffma2_rn(P.hy, superbee_diff2(back, __fadd2_rn(back, back), fwd, __fadd2_rn(fwd, fwd)), x);
        G[gedge_row + (P.own - y * A2)] = x;  // faces beyond the plane equal the edge value
    };
    // Iteration i (R = i mod 3).  Phase A: y faces of F row i (stage 1) and of
    // P row j = i-2 (stage 2) into the face rows of parity i, and F row
    // min(i+2, Nz) into the rotation (row Nz stays in its ring slot: nothing is
    // copied past the plane).  Then this thread's copy of row i+3 is waited
    // for and the block meets once: faces published, F row i+3 and P row i-1
    // visible.  Phase B: stage 1 on row i (z face of cell i+1, P(i) -- also
    // to shared memory -- and H(i)), stage 2 on row j (z face of cell j+1 from
    // P rows j .. i, the output row).  One barrier per row suffices: a face
    // row of parity i is rewritten only at iteration i+2, after every thread
    // has passed barrier i+1 and so finished iteration i; the F slot refilled
    // at iteration i held row i-2 and the P slot written held row i-4, both
    // last read before barrier i-1.  A row of F past the plane is not walked:
    // P(i) repeats the last predictor row.  FILL: issue the copy of row
    // i+PD+2 (every iteration that walks F).
    auto iter = [&](auto Rc, auto S1c, auto S2c, auto FILLc, int i) {
        constexpr int R = decltype(Rc)::value, R1 = (R + 1) % 3, R2 = (R + 2) % 3;
        constexpr bool st1 = decltype(S1c)::value != 0, st2 = decltype(S2c)::value != 0;
        constexpr bool do_fill = decltype(FILLc)::value != 0;
        float2* GF = Gb + (i & 1) * (2 * GS);
        float2* GP = GF + GS;
        const float2* Fi = Fr + (i & (RF - 1)) * RS;
        const float2* f2row = Fr + ((i + min(2, Nz - i)) & (RF - 1)) * RS;
        const float2* Pj = Pr + ((i - 2) & (RP - 1)) * RS;
#pragma unroll
        for (int k = 0; k < PT; ++k) {
            StreamPair& P = S[k];
            if (st1) {
                P.f[R2] = f2row[P.own];
                y_face(GF, Fi, P, P.f[R]);
            }
            if (st2) y_face(GP, Pj, P, P.p[R1]);
        }
        asm volatile("cp.async.wait_group %0;" ::"n"(PD - 2) : "memory");  // row i+3 of F landed
        __syncthreads();
        if (do_fill) fill(i + PD + 2);
        float2* Pw = Pr + (i & (RP - 1)) * RS;
#pragma unroll
        for (int k = 0; k < PT; ++k) {
            StreamPair& P = S[k];
            if (st1) {
                const float2 back = P.zf[R2], back2 = P.zf2[R2];
                P.zf[R] = sub2(P.f[R2], P.f[R1]);
                P.zf2[R] = __fadd2_rn(P.zf[R], P.zf[R]);
                const float2 gz_p = __ffma2_rn(P.hz, superbee_diff2(back, back2, P.zf[R], P.zf2[R]), P.f[R1]);
                const float2 dz = __fmul2_rn(P.wrz, P.dnz ? sub2(gz_p, P.gz[R]) : sub2(P.gz[R], P.gz[R2]));
                P.gz[R1] = gz_p;
                const float2 d = __fadd2_rn(__fmul2_rn(P.wry, sub2(GF[P.ghi], GF[P.glo])), dz);
                P.p[R] = max_lo2(__ffma2_rn(ndt, d, P.f[R]), lo);
                P.hh[R] = __ffma2_rn(nhdt, d, P.f[R]);
                Pw[P.own] = P.p[R];
            } else {
                P.p[R] = P.p[R2];
            }
        }
        if (st2) {
#pragma unroll
            for (int k = 0; k < PT; ++k) {
                StreamPair& P = S[k];
                const float2 back = P.pf[R2], back2 = P.pf2[R2];
                P.pf[R] = sub2(P.p[R], P.p[R2]);
                P.pf2[R] = __fadd2_rn(P.pf[R], P.pf[R]);
                const float2 gp_p = __ffma2_rn(P.hz, superbee_diff2(back, back2, P.pf[R], P.pf2[R]), P.p[R2]);
                const float2 dzp = __fmul2_rn(P.wrz, P.dnz ? sub2(gp_p, P.pz[R1]) : sub2(P.pz[R1], P.pz[R]));
                P.pz[R2] = gp_p;
                const float2 t = __ffma2_rn(nhdt, __fmul2_rn(P.wry, sub2(GP[P.ghi], GP[P.glo])), P.hh[R1]);
                const float2 v = max_lo2(__ffma2_rn(nhdt, dzp, t), lo);
                float* o = orow + 2 * (h + TPC * k);  // pair h + TPC k
                if (P.ok1) *reinterpret_cast<float2*>(o) = v;
                if (P.ok_half) *o = v.x;
            }
            orow += zs;
        }
    };

    for (int r = 0; r < PD + 2; ++r) fill(r);
    // rows 0 and 1: stage 1 only (row 1 is past a one-row plane when Nz = 0)
    asm volatile("cp.async.wait_group %0;" ::"n"(PD - 1) : "memory");  // rows 0 .. 2 landed
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PT; ++k) {
        StreamPair& P = S[k];
        P.f[0] = Fr[P.own];
        P.f[1] = Fr[(min(1, Nz) & (RF - 1)) * RS + P.own];
        P.gz[2] = P.gz[0] = P.f[0];  // faces of cells -1 and 0 of a clamped column: the edge value
        P.zf[2] = sub2(P.f[1], P.f[0]);
        P.zf2[2] = __fadd2_rn(P.zf[2], P.zf[2]);
    }
    iter(IntC<0>(), IntC<1>(), IntC<0>(), IntC<1>(), 0);
    if (Nz >= 1) iter(IntC<1>(), IntC<1>(), IntC<0>(), IntC<1>(), 1);
    else iter(IntC<1>(), IntC<0>(), IntC<0>(), IntC<1>(), 1);
#pragma unroll
    for (int k = 0; k < PT; ++k) {  // P rows 0 and 1 known: start the z-walk of P
        StreamPair& P = S[k];
        P.pz[2] = P.pz[0] = P.p[0];  // faces of cells -1 and 0
        P.pf[1] = sub2(P.p[1], P.p[0]);
        P.pf2[1] = __fadd2_rn(P.pf[1], P.pf[1]);
    }
    // rows 2 .. Nz: both stages, three rows per trip so the rotations stay in place
    int i = 2;
    if (i <= Nz) iter(IntC<2>(), IntC<1>(), IntC<1>(), IntC<1>(), i++);
#pragma unroll 1
    for (; i + 2 <= Nz; i += 3) {
        iter(IntC<0>(), IntC<1>(), IntC<1>(), IntC<1>(), i);
        iter(IntC<1>(), IntC<1>(), IntC<1>(), IntC<1>(), i + 1);
        iter(IntC<2>(), IntC<1>(), IntC<1>(), IntC<1>(), i + 2);
    }
    if (i <= Nz) iter(IntC<0>(), IntC<1>(), IntC<1>(), IntC<1>(), i++);
    if (i <= Nz) iter(IntC<1>(), IntC<1>(), IntC<1>(), IntC<1>(), i++);
    // rows past the plane: stage 2 only (the rows' phase is known only at run time)
    for (; i <= Nz + 2; ++i) {
        switch (i % 3) {
            case 0: iter(IntC<0>(), IntC<0>(), IntC<1>(), IntC<0>(), i); break;
            case 1: iter(IntC<1>(), IntC<0>(), IntC<1>(), IntC<0>(), i); break;
            default: iter(IntC<2>(), IntC<0>(), IntC<1>(), IntC<0>(), i); break;
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

__global__ void __maxnreg__(kStreamMaxReg) transport_stream_kernel(TransportArgs<float> a, int n_chunks) {
    transport_stream_body(a, n_chunks, blockIdx.x);
}

__global__ void __maxnreg__(kStreamMaxReg) transport_stream_slots_kernel(const TransportArgs<float>* __restrict__ args,
                                                                      const int* __restrict__ begin, int nslots,
                                                                      int n_chunks) {
    const int s = find_slot(begin, nslots, blockIdx.x);
    transport_stream_body(args[s], n_chunks, blockIdx.x - __ldg(begin + s));
}

int transport_stream_threads(int Ny) { return (Ny + 1) * kStreamTPC; }

bool transport_stream_supported(int Ny, int NA) {
    return NA % 2 == 0 && transport_stream_threads(Ny) <= kStreamMaxThreads &&
           transport_stream_smem(Ny + 1) <= 200 * 1024;
}

cudaError_t launch_transport_stream(const TransportArgs<float>& a, cudaStream_t s) {
    if (!a.pairs || !transport_stream_supported(a.Ny, a.NA)) return cudaErrorNotSupported;
    const int n_chunks = (a.NA + 2 * kStreamPairs - 1) / (2 * kStreamPairs);
    const size_t smem = transport_stream_smem(a.Ny + 1);
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void*>(transport_stream_kernel), smem);
    if (e != cudaSuccess) return e;
    const long long blocks = static_cast<long long>(a.Ng) * n_chunks;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    transport_stream_kernel<<<static_cast<unsigned>(blocks), transport_stream_threads(a.Ny), smem, s>>>(a, n_chunks);
    return cudaGetLastError();
}

cudaError_t launch_transport_stream_slots(const TransportArgs<float>* args, const int* begin, int nslots, int blocks,
                                          int Ny, int NA, cudaStream_t s) {
    if (nslots <= 0 || blocks <= 0) return cudaSuccess;
    if (!transport_stream_supported(Ny, NA)) return cudaErrorNotSupported;
    const int n_chunks = (NA + 2 * kStreamPairs - 1) / (2 * kStreamPairs);
    const size_t smem = transport_stream_smem(Ny + 1);
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void*>(transport_stream_slots_kernel), smem);
    if (e != cudaSuccess) return e;
    transport_stream_slots_kernel<<<blocks, transport_stream_threads(Ny), smem, s>>>(args, begin, nslots, n_chunks);
    return cudaGetLastError();
}

// The packed kernel applies when NA is even (8-byte aligned pairs) and the
// two angles of every pair share the signs of omega_y and omega_z.
bool transport_pairs_ok(const double* omega, int NA) {
    if (NA % 2 != 0) return false;
    for (int g = 0; g + 1 < NA; g += 2)
        if ((omega[2 * g] < 0) != (omega[2 * g + 2] < 0) || (omega[2 * g + 1] < 0) != (omega[2 * g + 3] < 0))
            return false;
    return true;
}

size_t transport_plane_smem(int NP, int ac, size_t elem) {
    return 2 * static_cast<size_t>(NP) * (NP | 1) * ac * elem;
}

template <typename T, int NP, int AC>
static cudaError_t launch_plane_np(const TransportArgs<T>& a, cudaStream_t s) {
    const int n_chunks = (a.NA + AC - 1) / AC;
    const size_t smem = transport_plane_smem(NP, AC, sizeof(T));
    auto kern = transport_plane_kernel<T, NP, AC>;
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
    if (e != cudaSuccess) return e;
    const long long blocks = static_cast<long long>(a.Ng) * n_chunks;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    kern<<<static_cast<unsigned>(blocks), (NP * AC + 31) / 32 * 32, smem, s>>>(a, n_chunks);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Large planes: the same unrolled walks over R x R regions, R = TT + 8.
// Block = (group, AC angles, one TT x TT output tile); its region is the tile
// plus a 4-cell halo, loaded with indices clamped to the plane, so cells
// outside the plane repeat the edge value -- exactly what the reference's
// clamped stencil indices read (the slope of a repeated triple is 0).  Every
// walk treats the region ends as line ends; that is wrong only within 2 cells
// of a region end that is not a plane edge, and the halo keeps those cells
// out of what the tile needs.  The predictor at out-of-plane cells is then
// replaced by its clamped in-plane value (the reference's stage 2 clamps its
// indices into P as well).  Output goes to a separate array (neighbouring
// tiles read this tile's input as their halo).
// ---------------------------------------------------------------------------
template <typename T, int R, int AC>
__global__ void __launch_bounds__((R * AC + 31) / 32 * 32) transport_tile_kernel(TransportArgs<T> a, int tiles_y,
                                                                                  int tiles_z, int n_chunks) {
    constexpr int TT = R - 8, N = R - 1, RP = R | 1, RS = RP * AC, PL = R * RS;
    constexpr int NT = (R * AC + 31) / 32 * 32;  // == blockDim.x
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* Fs = reinterpret_cast<T*>(smem_raw);
    T* Ps = Fs + PL;
    int b = blockIdx.x;
    const int tyi = b % tiles_y;
    b /= tiles_y;
    const int tzi = b % tiles_z;
    b /= tiles_z;
    const int chunk = b % n_chunks, ek = b / n_chunks;
    const int Ny = a.Ny, Nz = a.Nz, Ny1 = Ny + 1, NA = a.NA, a0 = chunk * AC;
    const int ry0 = tyi * TT - 4, rz0 = tzi * TT - 4;  // region origin (plane coordinates)
    const size_t plane = static_cast<size_t>(ek) * Ny1 * (Nz + 1) * NA + a0;
    const T* __restrict__ in = a.in + plane;
    T* __restrict__ out = a.out + plane;
    const int q = threadIdx.x % AC, line = threadIdx.x / AC;
    const bool qok = a0 + q < NA;
    const int ang = min(a0 + q, NA - 1);
    const T wy = a.omega[2 * ang], wz = a.omega[2 * ang + 1];
    const T wry = wy / a.dy, wrz = wz / a.dz;
    const bool dny = wy < T(0), dnz = wz < T(0);
    const T hy = dny ? T(-0.5) : T(0.5), hz = dnz ? T(-0.5) : T(0.5);
    const int sy = dny ? 1 : 0, sz = dnz ? 1 : 0;
    const T dt = a.dt, hdt = T(0.5) * a.dt;
    const T lo = a.preserve_sign ? -INFINITY : T(0);

    if (AC % Vec16<T>::W == 0 && NA % Vec16<T>::W == 0) {
        constexpr int W = Vec16<T>::W, NV = R * R * AC / W;
#pragma unroll 4
        for (int v = threadIdx.x; v < NV; v += NT) {
            const int e = v * W, aa = e % AC, p = e / AC;
            const int lz = p / R, ly = p - lz * R;
            const int gy = min(max(ry0 + ly, 0), Ny), gz = min(max(rz0 + lz, 0), Nz);
            const bool ok = a0 + aa < NA;
            cp_async16(Fs + lz * RS + ly * AC + aa, ok ? in + (static_cast<size_t>(gz) * Ny1 + gy) * NA + aa : in, ok);
        }
        cp_async_wait_all();
    } else {
#pragma unroll 4
        for (int e = threadIdx.x; e < R * R * AC; e += NT) {
            const int aa = e % AC, p = e / AC;
            const int lz = p / R, ly = p - lz * R;
            const int gy = min(max(ry0 + ly, 0), Ny), gz = min(max(rz0 + lz, 0), Nz);
            Fs[lz * RS + ly * AC + aa] = (a0 + aa < NA) ? in[(static_cast<size_t>(gz) * Ny1 + gy) * NA + aa] : T(0);
        }
    }
    __syncthreads();
    const bool act = line < R;
    // stage 1, y-part of div F (region rows) into Ps
    if (act) {
        const T* X = Fs + line * RS + q;
        T* D = Ps + line * RS + q - sy * AC;
        walk_plane_line<T, N, AC>(X, wry, hy, [&](int j, T d, T, T) { D[j * AC] = d; });
        Ps[line * RS + q + sy * N * AC] = T(0);
    }
    __syncthreads();
    // stage 1, z-part (region columns): predictor into Ps, H over F
    if (act) {
        T* Xc = Fs + line * AC + q;
        T* Pc = Ps + line * AC + q;
        T* Xe = Xc - sz * RS;
        T* Pe = Pc - sz * RS;
        walk_plane_line<T, N, RS>(Xc, wrz, hz, [&](int j, T dz, T xj, T xjm1) {
            const T f = dnz ? xjm1 : xj;
            const T d = Pe[j * RS] + dz;
            Pe[j * RS] = max(f - dt * d, lo);
            Xe[j * RS] = f - hdt * d;
        });
        const int cb = sz * N * RS;
        const T f = Xc[cb], d = Pc[cb];
        Pc[cb] = max(f - dt * d, lo);
        Xc[cb] = f - hdt * d;
    }
    __syncthreads();
    // the predictor outside the plane repeats its clamped in-plane value
    const bool edge = ry0 < 0 || rz0 < 0 || ry0 + R > Ny1 || rz0 + R > Nz + 1;
    if (edge) {
        for (int e = threadIdx.x; e < R * R * AC; e += NT) {
            const int aa = e % AC, p = e / AC;
            const int lz = p / R, ly = p - lz * R;
            const int cy = min(max(ry0 + ly, 0), Ny) - ry0, cz = min(max(rz0 + lz, 0), Nz) - rz0;
            if (cy != ly || cz != lz) Ps[lz * RS + ly * AC + aa] = Ps[cz * RS + cy * AC + aa];
        }
        __syncthreads();
    }
    // stage 2, y-part of div P on the tile's rows: H - dt/2 d_y P over F
    if (line < TT) {
        const int lz = line + 4;
        const T* X = Ps + lz * RS + q;
        T* Fe = Fs + lz * RS + q - sy * AC;
        walk_plane_line<T, N, AC>(X, wry, hy, [&](int j, T d, T, T) { Fe[j * AC] -= hdt * d; });
    }
    __syncthreads();
    // stage 2, z-part on the tile's columns and the corrector, to global
    const int gy = ry0 + 4 + line;
    if (line < TT && gy <= Ny) {
        const int ly = line + 4;
        const T* X = Ps + ly * AC + q;
        const T* Fc = Fs + ly * AC + q;
        const T* Fe = Fc - sz * RS;
        const size_t zs = static_cast<size_t>(Ny1) * NA;
        T* o = out + static_cast<size_t>(gy) * NA + q;  // + gz * zs
        const int gz_lo = rz0 + 4, gz_hi = min(rz0 + 4 + TT, Nz + 1);  // output rows of this tile
        walk_plane_line<T, N, RS>(X, wrz, hz, [&](int j, T d, T, T) {
            const int lz = j - sz, gz = rz0 + lz;
            if (qok && gz >= gz_lo && gz < gz_hi) o[static_cast<size_t>(gz) * zs] = max(Fe[j * RS] - hdt * d, lo);
        });
        const int lzb = sz * N, gzb = rz0 + lzb;  // the cell whose z-part is 0
        if (qok && gzb >= gz_lo && gzb < gz_hi) o[static_cast<size_t>(gzb) * zs] = max(Fc[lzb * RS], lo);
    }
}

size_t transport_tile_smem(int R, int ac, size_t elem) {
    return 2 * static_cast<size_t>(R) * (R | 1) * ac * elem;
}

constexpr int kTileRegion = 35;  // 27 x 27 output tiles

template <typename T, int AC>
static cudaError_t launch_tile_ac(const TransportArgs<T>& a, cudaStream_t s) {
    constexpr int R = kTileRegion, TT = R - 8;
    const int tiles_y = (a.Ny + 1 + TT - 1) / TT, tiles_z = (a.Nz + 1 + TT - 1) / TT;
    const int n_chunks = (a.NA + AC - 1) / AC;
    const size_t smem = transport_tile_smem(R, AC, sizeof(T));
    auto kern = transport_tile_kernel<T, R, AC>;
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
    if (e != cudaSuccess) return e;
    const long long blocks = static_cast<long long>(a.Ng) * n_chunks * tiles_y * tiles_z;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    kern<<<static_cast<unsigned>(blocks), (R * AC + 31) / 32 * 32, smem, s>>>(a, tiles_y, tiles_z, n_chunks);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_transport_tiles(const TransportArgs<T>& a, int ang_chunk, cudaStream_t s) {
    if (a.in == a.out) return cudaErrorInvalidValue;  // tiles read neighbours' input as halo
    if constexpr (sizeof(T) == 4) {
        if (ang_chunk == 4) return launch_tile_ac<T, 4>(a, s);
        if (ang_chunk == 8) return launch_tile_ac<T, 8>(a, s);
    } else {
        if (ang_chunk == 2) return launch_tile_ac<T, 2>(a, s);
        if (ang_chunk == 4) return launch_tile_ac<T, 4>(a, s);
    }
    return cudaErrorInvalidValue;
}

// Plane sizes (Ny+1 = Nz+1) and cluster sizes of the compiled cluster kernel
// (8 angles per plane chunk; bands of NP / CL rows).
#define BFPN_CLUSTER_PLANES(X) X(21, 2) X(41, 2) X(49, 4) X(65, 4) X(81, 4) X(97, 8) X(129, 8)

bool transport_cluster_supported(int Ny, int Nz) {
    if (Ny != Nz) return false;
    switch (Ny + 1) {
#define BFPN_CASE(NP, CL) case NP:
        BFPN_CLUSTER_PLANES(BFPN_CASE)
#undef BFPN_CASE
        return true;
        default: return false;
    }
}

template <int NP, int CL>
static cudaError_t launch_cluster_np(const TransportArgs<float>& a, cudaStream_t s) {
    constexpr int A2 = 4, AC = 2 * A2;
    using S = ClusterPlane<NP, CL, A2>;
    const int n_chunks = (a.NA + AC - 1) / AC;
    auto kern = transport_cluster_kernel<NP, CL, A2>;
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void*>(kern), S::smem);
    if (e != cudaSuccess) return e;
    const long long blocks = static_cast<long long>(a.Ng) * n_chunks * CL;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    kern<<<static_cast<unsigned>(blocks), S::NT, S::smem, s>>>(a, n_chunks);
    return cudaGetLastError();
}

cudaError_t launch_transport_cluster(const TransportArgs<float>& a, cudaStream_t s) {
    if (a.Ny != a.Nz || a.NA % 2 != 0 || !a.pairs) return cudaErrorNotSupported;
    switch (a.Ny + 1) {
#define BFPN_CASE(NP, CL) \
    case NP: return launch_cluster_np<NP, CL>(a, s);
        BFPN_CLUSTER_PLANES(BFPN_CASE)
#undef BFPN_CASE
        default: return cudaErrorNotSupported;
    }
}

// Plane sizes (Ny+1 = Nz+1) with a compiled whole-plane kernel.
#define BFPN_PLANE_SIZES(X) X(5) X(7) X(9) X(11) X(13) X(15) X(17) X(21) X(25) X(33)

bool transport_plane_supported(int Ny, int Nz) {
    if (Ny != Nz) return false;
    switch (Ny + 1) {
#define BFPN_CASE(NP) case NP:
        BFPN_PLANE_SIZES(BFPN_CASE)
#undef BFPN_CASE
        return true;
        default: return false;
    }
}

template <typename T, int AC>
static cudaError_t launch_plane_ac(const TransportArgs<T>& a, cudaStream_t s) {
    if (a.Ny != a.Nz) return cudaErrorNotSupported;
    switch (a.Ny + 1) {
#define BFPN_CASE(NP) \
    case NP: return launch_plane_np<T, NP, AC>(a, s);
        BFPN_PLANE_SIZES(BFPN_CASE)
#undef BFPN_CASE
        default: return cudaErrorNotSupported;
    }
}

template <int NP, int AC>
static cudaError_t launch_plane_f2_np(const TransportArgs<float>& a, cudaStream_t s) {
    const int n_chunks = (a.NA + AC - 1) / AC;
    const size_t smem = transport_plane_smem(NP, AC, sizeof(float));
    auto kern = transport_plane_f2_kernel<NP, AC>;
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
    if (e != cudaSuccess) return e;
    const long long blocks = static_cast<long long>(a.Ng) * n_chunks;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    kern<<<static_cast<unsigned>(blocks), (NP * AC / 2 + 31) / 32 * 32, smem, s>>>(a, n_chunks);
    return cudaGetLastError();
}

template <int AC>
static cudaError_t launch_plane_f2_ac(const TransportArgs<float>& a, cudaStream_t s) {
    if (a.Ny != a.Nz || a.NA % 2 != 0) return cudaErrorNotSupported;
    switch (a.Ny + 1) {
#define BFPN_CASE(NP) \
    case NP: return launch_plane_f2_np<NP, AC>(a, s);
        BFPN_PLANE_SIZES(BFPN_CASE)
#undef BFPN_CASE
        default: return cudaErrorNotSupported;
    }
}

template <typename T>
cudaError_t launch_transport_plane(const TransportArgs<T>& a, int ang_chunk, cudaStream_t s) {
    if constexpr (sizeof(T) == 4) {
        if (a.pairs && ang_chunk == 8) return launch_plane_f2_ac<8>(a, s);
        if (a.pairs && ang_chunk == 16) return launch_plane_f2_ac<16>(a, s);
        if (ang_chunk == 8) return launch_plane_ac<T, 8>(a, s);
        if (ang_chunk == 16) return launch_plane_ac<T, 16>(a, s);
    } else {
        if (ang_chunk == 4) return launch_plane_ac<T, 4>(a, s);
        if (ang_chunk == 8) return launch_plane_ac<T, 8>(a, s);
    }
    return cudaErrorInvalidValue;
}

// ---- multi-slot transport --------------------------------------------------
template <int NP, int AC>
static cudaError_t launch_plane_f2_slots(const TransportArgs<float>* args, const int* begin, int nslots, int blocks,
                                         int NA, cudaStream_t s) {
    const int n_chunks = (NA + AC - 1) / AC;
    const size_t smem = transport_plane_smem(NP, AC, sizeof(float));
    auto kern = transport_plane_f2_slots_kernel<NP, AC>;
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
    if (e != cudaSuccess) return e;
    kern<<<blocks, (NP * AC / 2 + 31) / 32 * 32, smem, s>>>(args, begin, nslots, n_chunks);
    return cudaGetLastError();
}

template <int NP, int CL>
static cudaError_t launch_cluster_slots(const TransportArgs<float>* args, const int* begin, int nslots, int blocks,
                                        int NA, cudaStream_t s) {
    constexpr int A2 = 4, AC = 2 * A2;
    using S = ClusterPlane<NP, CL, A2>;
    if (blocks % CL != 0) return cudaErrorInvalidValue;
    const int n_chunks = (NA + AC - 1) / AC;
    auto kern = transport_cluster_slots_kernel<NP, CL, A2>;
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void*>(kern), S::smem);
    if (e != cudaSuccess) return e;
    kern<<<blocks, S::NT, S::smem, s>>>(args, begin, nslots, n_chunks);
    return cudaGetLastError();
}

int transport_cluster_size(int NP) {
    switch (NP) {
#define BFPN_CASE(P, CL) \
    case P: return CL;
        BFPN_CLUSTER_PLANES(BFPN_CASE)
#undef BFPN_CASE
        default: return 0;
    }
}

cudaError_t launch_transport_slots(const TransportArgs<float>* args, const int* begin, int nslots, int blocks,
                                   int NP, int NA, int ang_chunk, bool cluster, cudaStream_t s) {
    if (nslots <= 0 || blocks <= 0) return cudaSuccess;
    if (NA % 2 != 0) return cudaErrorNotSupported;
    if (cluster) {
        switch (NP) {
#define BFPN_CASE(P, CL) \
    case P: return launch_cluster_slots<P, CL>(args, begin, nslots, blocks, NA, s);
            BFPN_CLUSTER_PLANES(BFPN_CASE)
#undef BFPN_CASE
            default: return cudaErrorNotSupported;
        }
    }
    switch (NP) {
#define BFPN_CASE(P)                                                                            \
    case P:                                                                                     \
        if (ang_chunk == 8) return launch_plane_f2_slots<P, 8>(args, begin, nslots, blocks, NA, s); \
        if (ang_chunk == 16) return launch_plane_f2_slots<P, 16>(args, begin, nslots, blocks, NA, s); \
        return cudaErrorInvalidValue;
        BFPN_PLANE_SIZES(BFPN_CASE)
#undef BFPN_CASE
        default: return cudaErrorNotSupported;
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
// Every entry sin(pi (m+1)(i+1) / (N+1)) is +- sin(pi k / (N+1)) for one
// k in 1..(N+1)/2, so the whole table is (N+1)/2 values held in registers;
// which value and which sign each FMA takes is fixed at compile time.
template <int N, typename T>
struct SineTable {
    T c[(N + 1) / 2];  // c[k-1] = sin(pi k / (N+1))
};

// Entry (m, i) of the DST-I matrix as (k, sign): the argument (m+1)(i+1) is
// reduced modulo 2(N+1); sin is 0 at 0 and N+1, negative on (N+1, 2(N+1)),
// and sin(pi b/(N+1)) = sin(pi (N+1-b)/(N+1)).
__host__ __device__ constexpr int sine_arg(int N, int m, int i) { return ((m + 1) * (i + 1)) % (2 * (N + 1)); }
__host__ __device__ constexpr int sine_k(int N, int m, int i) {
    const int a = sine_arg(N, m, i), b = a > N + 1 ? a - (N + 1) : a;
    return b < N + 1 - b ? b : N + 1 - b;
}
__host__ __device__ constexpr bool sine_neg(int N, int m, int i) { return sine_arg(N, m, i) > N + 1; }

// A product rounded on its own (never fused into a following add), so that
// every DST variant rounds the CN factor step the same way.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

template <int N, typename T>
__device__ __forceinline__ void dst1(const T (&c)[(N + 1) / 2], const T (&x)[N], T (&y)[N]) {
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
        const int n_terms = (m & 1) ? H : HC;
#pragma unroll
        for (int i = 0; i < n_terms; ++i) {
            const int k = sine_k(N, m, i);
            if (k == 0) continue;  // sin(pi) = 0: (m+1)(i+1) a multiple of N+1
            const T v = (m & 1) ? q[i] : p[i];
            acc = sine_neg(N, m, i) ? fma(-c[k - 1], v, acc) : fma(c[k - 1], v, acc);
        }
        y[m] = acc;
    }
}

template <int N, typename T>
__global__ void __launch_bounds__(256) angle_dst_kernel(AngleArgs<T> a, SineTable<N, T> S) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NA = N * N, RS = N + 1;  // padded row stride: conflict-free row and column access
    const int SL = a.slices_per_block;
    T* X = reinterpret_cast<T*>(smem_raw);
    T* Fac = X + SL * N * RS;  // CN factor rows of the (at most two) groups of this block's slices
    const long long total = static_cast<long long>(a.Ng) * a.nyz;
    const long long s0 = static_cast<long long>(blockIdx.x) * SL;
    const int ns = static_cast<int>(min(static_cast<long long>(SL), total - s0));
    const long long ek0 = s0 / a.nyz;
    const int split = static_cast<int>((ek0 + 1) * a.nyz - s0);  // first local slice of group ek0 + 1
    const int nrows = (split < ns && ek0 + 1 < a.Ng) ? 2 : 1;
    T* __restrict__ F = a.F + s0 * NA;
    // the block's slices are contiguous: element e of the run goes to row e / N
    // of the padded layout, i.e. to e + e / N
    constexpr int W = Vec16<T>::W;
    using V = typename Vec16<T>::type;
    if (NA % W == 0) {  // the run starts at s0 * NA: 16-byte aligned
#pragma unroll 4
        for (int v = threadIdx.x; v < ns * NA / W; v += 256) {
            const V val = reinterpret_cast<const V*>(F)[v];
            const T* t = reinterpret_cast<const T*>(&val);
#pragma unroll
            for (int k = 0; k < W; ++k) {
                const int e = v * W + k;
                X[e + e / N] = t[k];
            }
        }
    } else {
#pragma unroll 4
        for (int e = threadIdx.x; e < ns * NA; e += 256) X[e + e / N] = F[e];
    }
    for (int e = threadIdx.x; e < nrows * NA; e += 256) Fac[e] = a.fac[ek0 * NA + e];
    T c[(N + 1) / 2];
#pragma unroll
    for (int k = 0; k < (N + 1) / 2; ++k) c[k] = S.c[k];
    __syncthreads();
    T x[N], y[N];
    const int line = threadIdx.x;  // ns * N <= blockDim: one row / column per thread
    if (line < ns * N) {  // forward u
        T* R = X + line * RS;
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = R[k];
        dst1<N, T>(c, x, y);
#pragma unroll
        for (int k = 0; k < N; ++k) R[k] = y[k];
    }
    __syncthreads();
    if (line < ns * N) {  // forward v, factor, inverse v
        const int s = line / N, mu = line - s * N;
        T* C = X + s * N * RS + mu;
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = C[k * RS];
        dst1<N, T>(c, x, y);
        const T* fac = Fac + (s >= split ? NA : 0) + mu;
#pragma unroll
        for (int k = 0; k < N; ++k) y[k] = mul_rn(y[k], fac[k * N]);
        dst1<N, T>(c, y, x);
#pragma unroll
        for (int k = 0; k < N; ++k) C[k * RS] = x[k];
    }
    __syncthreads();
    if (line < ns * N) {  // inverse u
        T* R = X + line * RS;
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = R[k];
        dst1<N, T>(c, x, y);
#pragma unroll
        for (int k = 0; k < N; ++k) R[k] = y[k];
    }
    __syncthreads();
    if (NA % W == 0) {
#pragma unroll 4
        for (int v = threadIdx.x; v < ns * NA / W; v += 256) {
            V val;
            T* t = reinterpret_cast<T*>(&val);
#pragma unroll
            for (int k = 0; k < W; ++k) {
                const int e = v * W + k;
                t[k] = X[e + e / N];
            }
            reinterpret_cast<V*>(F)[v] = val;
        }
    } else {
#pragma unroll 4
        for (int e = threadIdx.x; e < ns * NA; e += 256) F[e] = X[e + e / N];
    }
}

// Pipelined form of the same transforms: persistent blocks walk their tiles
// (SL consecutive slices) through a ring of NST shared buffers.  Thread 0
// lands each tile with a bulk copy NST - 1 tiles ahead of its use and writes
// each finished tile back with a bulk store, so HBM traffic overlaps the
// transforms of the tiles in between.  Slices stay unpadded; rows move as
// 16-byte vectors when N * sizeof(T) allows.  Waits are bounded: on a
// timeout the block records an error code, drains its copies and stops.
template <int N, typename T, int NST>
__global__ void __launch_bounds__(256) angle_dst_pipe_kernel(AngleArgs<T> a, SineTable<N, T> S, long long n_tiles) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[NST];
    __shared__ int go;
    constexpr int NA = N * N;
    const int SL = a.slices_per_block, tid = threadIdx.x;
    const uint32_t stage_bytes = (static_cast<uint32_t>(SL) * NA * sizeof(T) + 127u) / 128u * 128u;
    const long long total = static_cast<long long>(a.Ng) * a.nyz;
    auto tile_of = [&](int i) { return static_cast<long long>(blockIdx.x) + static_cast<long long>(i) * gridDim.x; };
    auto nslices = [&](long long t) { return static_cast<int>(min(static_cast<long long>(SL), total - t * SL)); };
    auto buf = [&](int st) { return reinterpret_cast<T*>(smem_raw + st * stage_bytes); };
    int issued[NST] = {}, landed[NST] = {};  // thread 0's bookkeeping
    auto issue = [&](int i) {
        const long long t = tile_of(i);
        const int st = i % NST;
        const uint32_t bytes = static_cast<uint32_t>(nslices(t)) * NA * sizeof(T);
        mbar_expect_tx(&full[st], bytes);
        bulk_copy_g2s(buf(st), a.F + t * SL * NA, bytes, &full[st]);
        ++issued[st];
    };
    if (tid == 0) {
        for (int st = 0; st < NST; ++st) mbar_init(&full[st], 1);
        mbar_init_fence();
        for (int i = 0; i < NST - 1; ++i)
            if (tile_of(i) < n_tiles) issue(i);
        go = 1;
    }
    T c[(N + 1) / 2];
#pragma unroll
    for (int k = 0; k < (N + 1) / 2; ++k) c[k] = S.c[k];
    __syncthreads();
    T x[N], y[N];
    constexpr bool kVecRows = (N * sizeof(T)) % 16 == 0;
    using V = typename Vec16<T>::type;
    constexpr int W = Vec16<T>::W;
    auto load_row = [&](const T* R) {
        if constexpr (kVecRows) {
#pragma unroll
            for (int v = 0; v < N / W; ++v) {
                const V val = reinterpret_cast<const V*>(R)[v];
#pragma unroll
                for (int k = 0; k < W; ++k) x[v * W + k] = reinterpret_cast<const T*>(&val)[k];
            }
        } else {
#pragma unroll
            for (int k = 0; k < N; ++k) x[k] = R[k];
        }
    };
    auto store_row = [&](T* R) {
        if constexpr (kVecRows) {
#pragma unroll
            for (int v = 0; v < N / W; ++v) {
                V val;
#pragma unroll
                for (int k = 0; k < W; ++k) reinterpret_cast<T*>(&val)[k] = y[v * W + k];
                reinterpret_cast<V*>(R)[v] = val;
            }
        } else {
#pragma unroll
            for (int k = 0; k < N; ++k) R[k] = y[k];
        }
    };
    for (int i = 0;; ++i) {
        const long long t = tile_of(i);
        if (t >= n_tiles) break;
        const int st = i % NST;
        if (tid == 0) {
            if (tile_of(i + NST - 1) < n_tiles) {
                bulk_wait_read<0>();  // the store of tile i - 1 has left its stage
                issue(i + NST - 1);
            }
            const bool ok = mbar_wait(&full[st], (i / NST) & 1);
            if (ok) ++landed[st];
            go = ok ? 1 : 0;
        }
        __syncthreads();
        if (!go) break;
        T* X = buf(st);
        const int ns = nslices(t);
        const int line = tid;
        if (line < ns * N) {  // forward u
            load_row(X + line * N);
            dst1<N, T>(c, x, y);
            store_row(X + line * N);
        }
        __syncthreads();
        if (line < ns * N) {  // forward v, factor, inverse v
            const int sl = line / N, mu = line - sl * N;
            T* C = X + sl * NA + mu;
#pragma unroll
            for (int k = 0; k < N; ++k) x[k] = C[k * N];
            dst1<N, T>(c, x, y);
            const long long ek = (t * SL + sl) / a.nyz;
            const T* __restrict__ fac = a.fac + ek * NA + mu;
#pragma unroll
            for (int k = 0; k < N; ++k) y[k] = mul_rn(y[k], __ldg(fac + k * N));
            dst1<N, T>(c, y, x);
#pragma unroll
            for (int k = 0; k < N; ++k) C[k * N] = x[k];
        }
        __syncthreads();
        if (line < ns * N) {  // inverse u
            load_row(X + line * N);
            dst1<N, T>(c, x, y);
            store_row(X + line * N);
        }
        __syncthreads();
        if (tid == 0) {
            fence_proxy_async_smem();
            bulk_copy_s2g(a.F + t * SL * NA, X, static_cast<uint32_t>(ns) * NA * sizeof(T));
            bulk_commit();
        }
    }
    if (tid == 0) {
        if (!go) {
            atomicExch(a.err, 3);
            for (int st = 0; st < NST; ++st)
                if (issued[st] > landed[st]) mbar_wait(&full[st], (issued[st] - 1) & 1);
        }
        bulk_wait<0>();
    }
}

// DST-I of two lines at once (fp32x2): the scalar dst1's operations, pairwise.
template <int N>
__device__ __forceinline__ void dst1_pair(const float (&c)[(N + 1) / 2], const float2 (&x)[N], float2 (&y)[N]) {
    constexpr int H = N / 2, HC = (N + 1) / 2;
    float2 p[HC], q[H > 0 ? H : 1];
#pragma unroll
    for (int i = 0; i < H; ++i) {
        p[i] = __fadd2_rn(x[i], x[N - 1 - i]);
        q[i] = __ffma2_rn(x[N - 1 - i], make_float2(-1.f, -1.f), x[i]);
    }
    if (N & 1) p[H] = x[H];
#pragma unroll
    for (int m = 0; m < N; ++m) {
        float2 acc = make_float2(0.f, 0.f);
        const int n_terms = (m & 1) ? H : HC;
#pragma unroll
        for (int i = 0; i < n_terms; ++i) {
            const int k = sine_k(N, m, i);
            if (k == 0) continue;
            const float cc = sine_neg(N, m, i) ? -c[k - 1] : c[k - 1];
            acc = __ffma2_rn(make_float2(cc, cc), (m & 1) ? q[i] : p[i], acc);
        }
        y[m] = acc;
    }
}

// The pipelined DST for float state with two lines per thread: rows r and
// r + R/2 of a tile's R rows, then adjacent columns (mu, mu + 1) of a slice
// (N even).  128 threads per block, 2 * 128 / N slices per tile.
// Where work tile t lies: its slices in the state (F), their count, the
// first slice's index within its beam (for the group of each slice) and the
// beam's factor table and positions per group.
struct DstTile {
    float* F;
    int ns;
    long long slice0;
    const float* fac;
    int nyz;
};

// Tiles of one beam: SL consecutive slices each.
struct DstTilesOne {
    const AngleArgs<float>& a;
    int SL;
    __device__ DstTile operator()(long long t) const {
        const long long total = static_cast<long long>(a.Ng) * a.nyz;
        const int ns = static_cast<int>(min(static_cast<long long>(SL), total - t * SL));
        return DstTile{a.F + t * SL * a.Nom * a.Nmu, ns, t * SL, a.fac, a.nyz};
    }
};

// Tiles of the slots of a bundle: slot s owns tiles [tile_begin[s], tile_begin[s+1]).
struct DstTilesSlots {
    const AngleArgs<float>* args;
    const int* tile_begin;
    int nslots, SL;
    __device__ DstTile operator()(long long t) const {
        const int s = find_slot(tile_begin, nslots, t);
        const AngleArgs<float>& a = args[s];
        const long long lt = t - __ldg(tile_begin + s);
        const long long total = static_cast<long long>(a.Ng) * a.nyz;
        const int ns = static_cast<int>(min(static_cast<long long>(SL), total - lt * SL));
        return DstTile{a.F + lt * SL * a.Nom * a.Nmu, ns, lt * SL, a.fac, a.nyz};
    }
};

template <int N, int NST, typename Tiles>
__device__ __forceinline__ void angle_dst_pair_body(const Tiles& tiles, const SineTable<N, float>& S, int SL,
                                                    long long n_tiles, int* err) {
    static_assert(N % 2 == 0, "column pairs need an even N");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[NST];
    __shared__ int go;
    constexpr int NA = N * N, NH = N / 2;
    const int tid = threadIdx.x;
    const uint32_t stage_bytes = (static_cast<uint32_t>(SL) * NA * 4u + 127u) / 128u * 128u;
    auto tile_of = [&](int i) { return static_cast<long long>(blockIdx.x) + static_cast<long long>(i) * gridDim.x; };
    auto buf = [&](int st) { return reinterpret_cast<float*>(smem_raw + st * stage_bytes); };
    int issued[NST] = {}, landed[NST] = {};
    auto issue = [&](int i) {
        const DstTile d = tiles(tile_of(i));
        const int st = i % NST;
        const uint32_t bytes = static_cast<uint32_t>(d.ns) * NA * 4u;
        mbar_expect_tx(&full[st], bytes);
        bulk_copy_g2s(buf(st), d.F, bytes, &full[st]);
        ++issued[st];
    };
    if (tid == 0) {
        for (int st = 0; st < NST; ++st) mbar_init(&full[st], 1);
        mbar_init_fence();
        for (int i = 0; i < NST - 1; ++i)
            if (tile_of(i) < n_tiles) issue(i);
        go = 1;
    }
    float c[(N + 1) / 2];
#pragma unroll
    for (int k = 0; k < (N + 1) / 2; ++k) c[k] = S.c[k];
    __syncthreads();
    float2 x[N], y[N];
    constexpr bool kVecRows = (N * 4) % 16 == 0;
    auto load_rows = [&](const float* A, const float* B) {
        if constexpr (kVecRows) {
#pragma unroll
            for (int v = 0; v < N / 4; ++v) {
                const float4 u = reinterpret_cast<const float4*>(A)[v], w = reinterpret_cast<const float4*>(B)[v];
                x[4 * v] = make_float2(u.x, w.x);
                x[4 * v + 1] = make_float2(u.y, w.y);
                x[4 * v + 2] = make_float2(u.z, w.z);
                x[4 * v + 3] = make_float2(u.w, w.w);
            }
        } else {
#pragma unroll
            for (int k = 0; k < N; ++k) x[k] = make_float2(A[k], B[k]);
        }
    };
    auto store_rows = [&](float* A, float* B) {
        if constexpr (kVecRows) {
#pragma unroll
            for (int v = 0; v < N / 4; ++v) {
                reinterpret_cast<float4*>(A)[v] = make_float4(y[4 * v].x, y[4 * v + 1].x, y[4 * v + 2].x, y[4 * v + 3].x);
                reinterpret_cast<float4*>(B)[v] = make_float4(y[4 * v].y, y[4 * v + 1].y, y[4 * v + 2].y, y[4 * v + 3].y);
            }
        } else {
#pragma unroll
            for (int k = 0; k < N; ++k) {
                A[k] = y[k].x;
                B[k] = y[k].y;
            }
        }
    };
    for (int i = 0;; ++i) {
        const long long t = tile_of(i);
        if (t >= n_tiles) break;
        const int st = i % NST;
        if (tid == 0) {
            if (tile_of(i + NST - 1) < n_tiles) {
                bulk_wait_read<0>();  // the store of tile i - 1 has left its stage
                issue(i + NST - 1);
            }
            const bool ok = mbar_wait(&full[st], (i / NST) & 1);
            if (ok) ++landed[st];
            go = ok ? 1 : 0;
        }
        __syncthreads();
        if (!go) break;
        float* X = buf(st);
        const DstTile d = tiles(t);
        const int ns = d.ns, half = ns * NH;  // row pairs = column pairs = ns * N / 2
        if (tid < half) {  // forward u on rows tid and tid + half
            load_rows(X + tid * N, X + (tid + half) * N);
            dst1_pair<N>(c, x, y);
            store_rows(X + tid * N, X + (tid + half) * N);
        }
        __syncthreads();
        if (tid < half) {  // forward v, factor, inverse v on columns (mu, mu + 1)
            const int sl = tid / NH, mu = 2 * (tid - sl * NH);
            float2* C = reinterpret_cast<float2*>(X + sl * NA + mu);
#pragma unroll
            for (int k = 0; k < N; ++k) x[k] = C[k * NH];
            dst1_pair<N>(c, x, y);
            const long long ek = (d.slice0 + sl) / d.nyz;
            const float2* __restrict__ fac = reinterpret_cast<const float2*>(d.fac + ek * NA + mu);
#pragma unroll
            for (int k = 0; k < N; ++k) y[k] = __fmul2_rn(y[k], __ldg(fac + k * NH));
            dst1_pair<N>(c, y, x);
#pragma unroll
            for (int k = 0; k < N; ++k) C[k * NH] = x[k];
        }
        __syncthreads();
        if (tid < half) {  // inverse u
            load_rows(X + tid * N, X + (tid + half) * N);
            dst1_pair<N>(c, x, y);
            store_rows(X + tid * N, X + (tid + half) * N);
        }
        __syncthreads();
        if (tid == 0) {
            fence_proxy_async_smem();
            bulk_copy_s2g(d.F, X, static_cast<uint32_t>(ns) * NA * 4u);
            bulk_commit();
        }
    }
    if (tid == 0) {
        if (!go) {
            atomicExch(err, 3);
            for (int st = 0; st < NST; ++st)
                if (issued[st] > landed[st]) mbar_wait(&full[st], (issued[st] - 1) & 1);
        }
        bulk_wait<0>();
    }
}

template <int N, int NST>
__global__ void __launch_bounds__(128) angle_dst_pair_kernel(AngleArgs<float> a, SineTable<N, float> S,
                                                             long long n_tiles) {
    angle_dst_pair_body<N, NST>(DstTilesOne{a, a.slices_per_block}, S, a.slices_per_block, n_tiles, a.err);
}

// The slots' tiles in one persistent launch; the error word is slot 0's.
template <int N, int NST>
__global__ void __launch_bounds__(128) angle_dst_pair_slots_kernel(const AngleArgs<float>* __restrict__ args,
                                                                   const int* __restrict__ tile_begin, int nslots,
                                                                   SineTable<N, float> S, int SL, long long n_tiles) {
    angle_dst_pair_body<N, NST>(DstTilesSlots{args, tile_begin, nslots, SL}, S, SL, n_tiles, args[0].err);
}

template <int N, typename T>
static cudaError_t launch_angle_dst(const AngleArgs<T>& a, cudaStream_t s) {
    SineTable<N, T> S;
    // sine_u lives on the device; the distinct values are built from the same
    // formula the tables use (angle_diffusion.cu:393-397)
    for (int k = 1; k <= (N + 1) / 2; ++k)
        S.c[k - 1] = static_cast<T>(std::sin(3.14159265358979323846 * k / (N + 1)));
    const int SL = std::max(1, std::min(256 / N, a.nyz));  // at most two groups per block
    const long long total = static_cast<long long>(a.Ng) * a.nyz;
    const long long n_tiles = (total + SL - 1) / SL;
    if constexpr (sizeof(T) == 4 && N % 2 == 0 && N >= 4) {
        if (a.err && a.pairs) {  // two lines per thread, 128 threads: 2 * 128 / N slices per tile
            constexpr int NST = 2, SLP = 256 / N;  // 2 stages: 5 blocks per SM at N = 20
            const int SL2 = std::max(1, std::min(SLP, a.nyz));
            const long long tiles2 = (total + SL2 - 1) / SL2;
            const size_t stage = (static_cast<size_t>(SL2) * N * N * 4 + 127) / 128 * 128;
            auto pk = angle_dst_pair_kernel<N, NST>;
            cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void*>(pk), NST * stage);
            if (e != cudaSuccess) return e;
            int dev = 0, sms = 0, per_sm = 0;
            if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
            if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
            if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pk, 128, NST * stage)) != cudaSuccess)
                return e;
            AngleArgs<T> b = a;
            b.slices_per_block = SL2;
            const long long grid = std::min<long long>(tiles2, static_cast<long long>(sms) * std::max(per_sm, 1));
            pk<<<static_cast<unsigned>(grid), 128, NST * stage, s>>>(b, S, tiles2);
            return cudaGetLastError();
        }
    }
    if (a.err && (N * N) % Vec16<T>::W == 0) {
        // pipelined: 2 stages of whole tiles per block (more blocks per SM beat deeper rings)
        constexpr int NST = 2;
        const size_t stage = (static_cast<size_t>(SL) * N * N * sizeof(T) + 127) / 128 * 128;
        auto pk = angle_dst_pipe_kernel<N, T, NST>;
        cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void*>(pk), NST * stage);
        if (e != cudaSuccess) return e;
        int dev = 0, sms = 0, per_sm = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pk, 256, NST * stage)) != cudaSuccess)
            return e;
        AngleArgs<T> b = a;
        b.slices_per_block = SL;
        const long long grid = std::min<long long>(n_tiles, static_cast<long long>(sms) * std::max(per_sm, 1));
        pk<<<static_cast<unsigned>(grid), 256, NST * stage, s>>>(b, S, n_tiles);
        return cudaGetLastError();
    }
    const size_t smem = (static_cast<size_t>(SL) * N * (N + 1) + 2 * static_cast<size_t>(N) * N) * sizeof(T);
    auto kern = angle_dst_kernel<N, T>;
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
    if (e != cudaSuccess) return e;
    AngleArgs<T> b = a;
    b.slices_per_block = SL;
    if (n_tiles > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    kern<<<static_cast<unsigned>(n_tiles), 256, smem, s>>>(b, S);
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

// ---- multi-slot DST ---------------------------------------------------------
int angle_slots_tile(int N) { return 256 / N; }

template <int N, int NST>
static cudaError_t launch_angle_slots_n(const AngleArgs<float>* args, const int* tile_begin, int nslots,
                                        long long tiles, cudaStream_t s) {
    SineTable<N, float> S;
    for (int k = 1; k <= (N + 1) / 2; ++k)
        S.c[k - 1] = static_cast<float>(std::sin(3.14159265358979323846 * k / (N + 1)));
    const int SL = angle_slots_tile(N);
    const size_t stage = (static_cast<size_t>(SL) * N * N * 4 + 127) / 128 * 128;
    auto pk = angle_dst_pair_slots_kernel<N, NST>;
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void*>(pk), NST * stage);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pk, 128, NST * stage)) != cudaSuccess) return e;
    const long long grid = std::min<long long>(tiles, static_cast<long long>(sms) * std::max(per_sm, 1));
    pk<<<static_cast<unsigned>(grid), 128, NST * stage, s>>>(args, tile_begin, nslots, S, SL, tiles);
    return cudaGetLastError();
}

cudaError_t launch_angle_slots(const AngleArgs<float>* args, const int* tile_begin, int nslots, long long tiles,
                               int N, int stages, cudaStream_t s) {
    if (nslots <= 0 || tiles <= 0) return cudaSuccess;
    if (stages != 2 && stages != 3) return cudaErrorInvalidValue;
    switch (N) {
#define BFPN_DST_SLOTS(n)                                                                   \
    case n:                                                                                 \
        return stages == 2 ? launch_angle_slots_n<n, 2>(args, tile_begin, nslots, tiles, s) \
                           : launch_angle_slots_n<n, 3>(args, tile_begin, nslots, tiles, s);
        BFPN_DST_SLOTS(4) BFPN_DST_SLOTS(6) BFPN_DST_SLOTS(8) BFPN_DST_SLOTS(10) BFPN_DST_SLOTS(12)
        BFPN_DST_SLOTS(14) BFPN_DST_SLOTS(16) BFPN_DST_SLOTS(18) BFPN_DST_SLOTS(20) BFPN_DST_SLOTS(22)
        BFPN_DST_SLOTS(24) BFPN_DST_SLOTS(28) BFPN_DST_SLOTS(32)
#undef BFPN_DST_SLOTS
        default: return cudaErrorNotSupported;
    }
}

template <typename T>
cudaError_t launch_angle_generic(const AngleArgs<T>& a, cudaStream_t s) {
    const int NA = a.Nom * a.Nmu;
    const size_t smem = (static_cast<size_t>(a.Nom) * a.Nom + static_cast<size_t>(a.Nmu) * a.Nmu
                         + 2 * static_cast<size_t>(a.slices_per_block) * NA) * sizeof(T);
    auto kern = angle_kernel<T>;
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
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
            const double y = f ? static_cast<double>(f[ek * lanes + lane]) : 0.0;  // f = nullptr: psi^1 only
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

// One block per slot of a bundle: launch_finalize_idd's reduction with the slot's arguments.
__global__ void __launch_bounds__(1024) finalize_idd_slots_kernel(const IddFinalArgs* __restrict__ args) {
    const IddFinalArgs& f = args[blockIdx.x];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < f.n; i += blockDim.x) { a += f.p[2 * i]; b += f.p[2 * i + 1]; }
    for (int i = threadIdx.x; i < f.n2; i += blockDim.x) a += f.p2[2 * i];
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
            const int c = *f.counter;
            if (c >= 0 && c < f.capacity) {
                f.hist_idd[c] = a * f.idd_scale;
                f.hist_proxy[c] = b * f.proxy_scale;
            }
            *f.counter = c + 1;
        }
    }
}

cudaError_t launch_finalize_idd_slots(const IddFinalArgs* args, int nslots, cudaStream_t s) {
    if (nslots <= 0) return cudaSuccess;
    finalize_idd_slots_kernel<<<nslots, 1024, 0, s>>>(args);
    return cudaGetLastError();
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

// YZ dose plane (spotDosePlaneKernel, bfpm_solver.cu:433-475): per position,
// the Eq. 24 dose of primary + secondary summed over groups and angles,
// times du dv.  One block per position; dose_coef holds the per-group weights
// already divided by the density.
template <typename T>
__global__ void __launch_bounds__(256) spot_plane_kernel(const T* F, const T* f, const T* F1, const T* f1,
                                                         const double* __restrict__ dc, int Ng, int nyz, int NA,
                                                         double dudv, double* plane) {
    const int pos = blockIdx.x;
    const long long per_e = static_cast<long long>(nyz) * NA;
    double acc = 0.0;
    for (int e = threadIdx.x; e < Ng * NA; e += blockDim.x) {
        const int ek = e / NA, a = e - ek * NA;
        const long long i = ek * per_e + static_cast<long long>(pos) * NA + a;
        const double p1 = static_cast<double>(F[i]) + static_cast<double>(F1[i]);
        const double p2 = static_cast<double>(f[i]) + static_cast<double>(f1[i]);
        acc += dc[2 * ek] * p1 + dc[2 * ek + 1] * p2;
    }
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = acc;
    __syncthreads();
    if (w == 0) {
        acc = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (l == 0) plane[pos] = acc * dudv;
    }
}

template <typename T>
cudaError_t launch_spot_plane(const T* F, const T* f, const T* F1, const T* f1, const double* dc, int Ng, int nyz,
                              int NA, double dudv, double* plane, cudaStream_t s) {
    spot_plane_kernel<T><<<nyz, 256, 0, s>>>(F, f, F1, f1, dc, Ng, nyz, NA, dudv, plane);
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
    template cudaError_t launch_lite_energy<T>(T*, const double*, double, int, long long, const double*, int, int,  \
                                               int, int, double*, cudaStream_t);                                  \
    template cudaError_t launch_transport<T>(const TransportArgs<T>&, int, cudaStream_t);                         \
    template cudaError_t launch_transport_plane<T>(const TransportArgs<T>&, int, cudaStream_t);                   \
    template cudaError_t launch_transport_tiles<T>(const TransportArgs<T>&, int, cudaStream_t);                   \
    template cudaError_t launch_angle<T>(const AngleArgs<T>&, cudaStream_t);                                      \
    template cudaError_t launch_idd_partials<T>(const T*, const T*, const double*, int, long long, int, int, int,  \
                                                int, int, double*, int, cudaStream_t);                            \
    template cudaError_t launch_energy_moments<T>(const T*, const T*, const T*, const T*, int, long long, double, \
                                                  double*, cudaStream_t);                                         \
    template cudaError_t launch_init_beam<T>(T*, const double*, const double*, long long, int, cudaStream_t);      \
    template cudaError_t launch_spot_plane<T>(const T*, const T*, const T*, const T*, const double*, int, int, int, \
                                              double, double*, cudaStream_t);

BFPN_INSTANTIATE(double)
BFPN_INSTANTIATE(float)
template cudaError_t launch_convert<double, float>(const double*, float*, long long, cudaStream_t);
template cudaError_t launch_convert<float, double>(const float*, double*, long long, cudaStream_t);
template cudaError_t launch_convert<double, double>(const double*, double*, long long, cudaStream_t);

}  // namespace bfpn
