// Host-side physics tables of one beam (the set-up half of the reference's
// BFPnSolver::initialize, bfpm_solver.cu:1435-2026).  Built once per beam on
// the host in double precision, then uploaded.
#pragma once

#include "../../include/bfpn_capi.h"

#include <cstddef>
#include <functional>
#include <new>
#include <string>
#include <utility>
#include <vector>

namespace bfpn {

// Allocator whose new elements are left uninitialised: a large table is first
// written (and so first touched) by the threads that fill it, instead of
// being zeroed page by page on one thread beforehand.
template <typename T>
struct UninitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = UninitAlloc<U>;
    };
    UninitAlloc() = default;
    template <typename U>
    UninitAlloc(const UninitAlloc<U>&) noexcept {}
    template <typename U>
    void construct(U* p) noexcept {
        ::new (static_cast<void*>(p)) U;
    }
    template <typename U, typename... A>
    void construct(U* p, A&&... args) {
        ::new (static_cast<void*>(p)) U(std::forward<A>(args)...);
    }
};
using HostTable = std::vector<double, UninitAlloc<double>>;

// Runs f(begin, end) over [0, n) split into contiguous ranges, one per host
// thread (up to 32); one call on the caller's thread when n < min_per_thread.
void parallel_ranges(size_t n, size_t min_per_thread, const std::function<void(size_t, size_t)>& f);

struct Deltas {
    double dt, dy, dz, dg, du, dv;
};

// GridParams::computeDeltas (bfpm_solver.cu:1116-1127).
Deltas compute_deltas(const bfpn_grid& g);

struct BeamTables {
    int Ng = 0, Ny = 0, Nz = 0, Nmu = 0, Nom = 0, nyz = 0, NA = 0;
    Deltas d{};
    std::vector<double> mu;        // Ng x 3, zero rows past the file
    std::vector<double> sigma;     // Ng, after the optional legacy calibration
    std::vector<double> S_s;       // Ng + 1
    std::vector<double> T_c;       // Ng
    std::vector<double> sig_trg;   // Ng
    std::vector<double> en;        // Ng + 1
    std::vector<double> omega;     // NA x 2 (omega_y, omega_z)
    std::vector<double> ker_e1, ker_e2;  // Ng x Ng, row = output group, column = source group
    std::vector<int> band_begin, band_end;  // per output group
    HostTable ker_v;               // Ng x NA x NA, [src][in][out]; empty when built as float only
    std::vector<float, UninitAlloc<float>> ker_v_f;  // the same table rounded to float (float-state contexts)
    std::vector<double> sine_u, sine_v;     // Nom x Nom, Nmu x Nmu
    std::vector<double> beam_yza;  // nyz x NA  (initial-beam transverse/angular factor)
    std::vector<double> beam_e;    // Ng        (initial-beam energy factor)
    double omega_center_y = 0.0, omega_center_z = 0.0;
    double spatial_mass = 0.0, angular_mass = 0.0, energy_mass = 0.0, initial_scale = 1.0;
    int mu_rows = 0;
};

// Builds every table; returns false with a message on invalid input
// (mirrors the reference's runtime_error cases).
// float_kernel: the angular kernel is built as ker_v_f (the float rounding of
// each double entry) instead of ker_v.
bool build_tables(const bfpn_grid& g, const bfpn_phys& p, const double* mu, int mu_rows, const double* sigma,
                  int sigma_rows, BeamTables& t, std::string& err, bool float_kernel = false);

// ker_v in double, built on first use when the tables were built float only.
const HostTable& angular_kernel_f64(BeamTables& t);

// Energy-sweep constants [Ng][kEnergyCoef] for half-step dt (see common.cuh).
std::vector<double> energy_coefficients(const BeamTables& t, const bfpn_phys& p, double dt);

// Eq. 24 dose weights [Ng][2] of psi^1 and psi^2, divided by the density;
// the quadrature du dv dy dz is applied at the end of the reduction.
std::vector<double> dose_coefficients(const BeamTables& t, const bfpn_phys& p);

// Lite-memory step constants per group (litePrimaryEnergyStepKernel,
// bfpm_solver.cu:607-619): [2*ek] = max(S_s[ek+1],0) / dg and
// [2*ek+1] = max(1/dt + max(S_s[ek],0)/dg + max(sigma_c[ek],0), eps).
std::vector<double> lite_coefficients(const BeamTables& t, double dt);

// Crank-Nicolson DST-I factor [Ng][NA] for step dt (buildDiffusionFactorKernel
// times the 4/((Nom+1)(Nmu+1)) normalisation).
std::vector<double> angle_factor(const BeamTables& t, const bfpn_phys& p, double dt);

// Reads the first Ng rows of the two table files as the reference does
// (bfpm_solver.cu:1435-1480).  Returns false and sets err when a file is
// missing.
bool read_table_files(const std::string& data_path, int Ng, std::vector<double>& mu, int& mu_rows,
                      std::vector<double>& sigma, int& sigma_rows, std::string& mu_path, std::string& err);

}  // namespace bfpn
