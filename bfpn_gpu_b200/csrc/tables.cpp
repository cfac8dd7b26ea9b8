// Host-side physics tables of one beam.  Compiled without floating-point
// contraction so every table equals, bit for bit, the one the reference's
// host code builds from the same inputs.  Citations are to the reference
// (xiaojin1423764/BFPn_GPU) file:line whose arithmetic each builder keeps.

#include "tables.hpp"
#include "common.cuh"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <atomic>
#include <cstdint>
#include <limits>
#include <thread>

namespace bfpn {
namespace {

constexpr double kPi = 3.14159265358979323846;  // include/config.hpp:9
constexpr double kElectronMass = 9.10956e-31;   // config.hpp:10
constexpr double kProtonMass = 1.673e-27;       // config.hpp:11
constexpr double kAlpha = 1.0 / 137.0;          // config.hpp:12
constexpr double kLight = 2.998e8;              // config.hpp:13
constexpr double kHbarC = 197.3;                // config.hpp:14
constexpr double kMeVToJ = 1.6e-13;             // config.hpp:17
constexpr double kKernelThreshold = 1e-3;       // config.hpp:40
constexpr double kSparseThreshold = 1e-5;       // config.hpp:41

struct Fraction {
    int Z;
    double weight;
};

// Mass fractions of the three material presets (bfpm_solver.cu:184-196).
std::vector<Fraction> material_fractions(int material) {
    switch (material) {
        case BFPN_MATERIAL_BONE:
            return {{1, 0.04200}, {6, 0.1940}, {7, 0.04000}, {8, 0.4250}, {11, 0.001000},
                    {12, 0.002000}, {15, 0.09200}, {16, 0.003000}, {20, 0.2010}};
        case BFPN_MATERIAL_AIR:
            return {{6, 0.0001248}, {7, 0.7553}, {8, 0.2318}, {18, 0.01283}};
        default:
            return {{1, 0.1111}, {8, 0.8889}};
    }
}

// Mean excitation energy in eV (bfpm_solver.cu:150-154).
double excitation_ev(int Z) {
    return Z == 1 ? 19.0 : (Z <= 13 ? 11.2 + 11.7 * Z : 52.8 + 8.71 * Z);
}

// Mass number used by the Bethe ratio (bfpm_solver.cu:156-170).
double mass_number(int Z) {
    static const int zs[] = {1, 6, 7, 8, 11, 12, 15, 16, 18, 20};
    static const double as[] = {1.0, 12.0, 14.0, 16.0, 23.0, 24.0, 31.0, 32.0, 40.0, 40.0};
    for (int i = 0; i < 10; ++i)
        if (zs[i] == Z) return as[i];
    return 2.0 * Z;
}

// Bethe mass stopping power of one element (bfpm_solver.cu:172-182).
double bethe(double E, int Z) {
    const double kappa = 0.307;
    const double me_c2 = 0.51099895e6;
    double beta2 = std::max(E * (E + 2.0 * 938.3) / ((E + 938.3) * (E + 938.3)), kEpsilon);
    double gamma2 = 1.0 / std::max(1.0 - beta2, kEpsilon);
    double arg = std::max(2.0 * me_c2 * beta2 * gamma2 / excitation_ev(Z), 1.0 + kEpsilon);
    double bracket = std::log(arg) - beta2;
    return kappa * (static_cast<double>(Z) / mass_number(Z)) / beta2 * bracket;
}

double weighted_bethe(const std::vector<Fraction>& mix, double E) {
    double s = 0.0;
    for (const Fraction& f : mix) s += f.weight * bethe(E, f.Z);
    return s;
}

// Stopping power at the DG nodes (computeStoppingPower, bfpm_solver.cu:1570-1597):
// the legacy water fit scaled by the Bethe ratio material/water.  Node 0 is
// at 1 MeV, node Ng at Lg+1, the others at group midpoints below the node.
void stopping_power(const bfpn_grid& g, int material, double dg, std::vector<double>& S) {
    const auto mix = material_fractions(material);
    const auto water = material_fractions(BFPN_MATERIAL_WATER);
    S.resize(g.Ng + 1);
    for (int i = 0; i <= g.Ng; ++i) {
        const double E = (i == 0) ? 1.0 : (i == g.Ng) ? g.Lg + 1.0 : (i - 0.5) * dg + 1.0;
        const double wm = weighted_bethe(mix, E);
        const double ww = weighted_bethe(water, E);
        const double beta_2 = E * (E + 2.0 * 938.3) / std::pow(E + 938.3, 2);
        const double F_beta = std::log(1.02e6 * beta_2 / (1.0 - beta_2)) - beta_2 - 4.31;
        const double water_fit = 0.170 / beta_2 * F_beta + 0.02;
        S[i] = water_fit * ((ww > kEpsilon) ? wm / ww : 1.0);
    }
}

// Straggling coefficient (computeStraggling, bfpm_solver.cu:1599-1615): the
// reference's simplified formula is energy independent.
void straggling(int Ng, std::vector<double>& T) {
    const double eta = 8.99e18 * 4.0 * kPi * std::pow(1.6e-19, 4) / std::pow(1.6e-13, 2) / 100.0;
    T.assign(Ng, eta * 3.34e29 * 1.2);
}

// Transport cross-section (computeTransportCrossSection, bfpm_solver.cu:1617-1636).
void transport_cross_section(int Ng, double dg, std::vector<double>& sig) {
    sig.resize(Ng);
    for (int i = 0; i < Ng; ++i) {
        const double E = (i + 0.5) * dg + 1.0;
        const double beta = std::sqrt(2.0 * E * kMeVToJ / kProtonMass) / (3.0 * kLight);
        const double Zt = 3;
        const double eta = std::pow(Zt, 2.0 / 3.0) * std::pow(kAlpha, 2) * std::pow(kElectronMass / kProtonMass, 2)
                           / (beta * beta);
        const double mid = std::log((eta + 1.0) / eta) - 1.0 / (eta + 1.0);
        sig[i] = 2.0 * kPi * 3.34 * std::pow(kHbarC, 2) * std::pow(kAlpha, 2) / 4.0 * Zt * Zt / (E * E) * mid / 1000.0;
    }
}

// Catastrophic energy kernels (initializeKernels, bfpm_solver.cu:1638-1721).
// The exponential transfer kernel of source group j into lower groups is
// shifted one group, flipped to high-energy-first order, thresholded, scaled
// by sigma_c of the source column, and split into the DG pair
// e1 = (k_row + k_row+1)/2, e2 = (k_row+1 - k_row)/2.
void energy_kernels(BeamTables& t) {
    const int Ng = t.Ng;
    const double dg = t.d.dg;
    const size_t NN = static_cast<size_t>(Ng) * Ng;
    // transfer[i][j]: from group j to group i >= j, before the shift
    std::vector<double> transfer(NN, 0.0);
    for (int j = 0; j < Ng - 1; ++j) {
        const double mu3 = t.mu[j * 3 + 2];
        if (mu3 == 0) continue;
        for (int i = j; i < Ng - 1; ++i) transfer[i * Ng + j] = dg / mu3 * std::exp(-(i - j + 0.5) * dg / mu3);
    }
    std::vector<double> ker_e(NN, 0.0);
    for (int row = 0; row < Ng; ++row) {
        for (int col = 0; col < Ng; ++col) {
            // flipped indices into the shifted kernel: shifted[i][j] = transfer[i-1][j] for i > j
            const int i = Ng - 1 - row, j = Ng - 1 - col;
            double value = 0.0;
            if (j < Ng - 1 && i > j) value = transfer[(i - 1) * Ng + j];
            if (std::abs(value) < kSparseThreshold) value = 0.0;
            ker_e[row * Ng + col] = value * t.sigma[col];
        }
    }
    t.ker_e1.assign(NN, 0.0);
    t.ker_e2.assign(NN, 0.0);
    for (int row = 0; row < Ng; ++row)
        for (int col = 0; col < Ng; ++col) {
            const double cur = ker_e[row * Ng + col];
            const double next = (row + 1 < Ng) ? ker_e[(row + 1) * Ng + col] : 0.0;
            t.ker_e1[row * Ng + col] = 0.5 * (cur + next);
            t.ker_e2[row * Ng + col] = 0.5 * (-cur + next);
        }
    t.band_begin.assign(Ng, 0);
    t.band_end.assign(Ng, 0);
    for (int row = 0; row < Ng; ++row) {
        int b = Ng, e = 0;
        for (int col = 0; col < Ng; ++col)
            if (t.ker_e1[row * Ng + col] != 0.0 || t.ker_e2[row * Ng + col] != 0.0) {
                b = std::min(b, col);
                e = std::max(e, col + 1);
            }
        if (b < Ng) {
            t.band_begin[row] = b;
            t.band_end[row] = e;
        }
    }
}

// Angular scattering kernel (bfpm_solver.cu:1723-1790): for each source group
// with mu1, mu2 != 0, a column-normalised theta^(mu1-1) exp(-theta/mu2)
// (1+|w_in|^2)^-1.5 over the input directions, entries below 1e-3 after
// normalisation dropped.  The last group carries no kernel.
//
// Same values as the reference's loop, built faster: theta(in, out) takes far
// fewer distinct values than NA^2 (it is symmetric bit for bit, and shifted
// direction pairs repeat), so theta^(mu1-1) exp(-theta/mu2) is evaluated once
// per distinct value and group; the rows are then filled in memory order,
// each column sum still adding its inputs in increasing order.  Groups are
// spread over the host's threads, and each thread is the first to touch the
// table pages it fills.
void angular_kernel(BeamTables& t, bool as_float) {
    const int NA = t.NA, Ng = t.Ng;
    const size_t NA2 = static_cast<size_t>(NA) * NA;
    std::vector<double> theta(NA2);  // [in][out], degrees; rows of inputs over the host's threads
    parallel_ranges(NA, 64, [&](size_t in0, size_t in1) {
        for (size_t in = in0; in < in1; ++in) {
            const double iy = t.omega[2 * in], iz = t.omega[2 * in + 1];
            const double inn = std::sqrt(1.0 + iy * iy + iz * iz);
            for (int out = 0; out < NA; ++out) {
                const double oy = t.omega[2 * out], oz = t.omega[2 * out + 1];
                const double on = std::sqrt(1.0 + oy * oy + oz * oz);
                double c = (1.0 + iy * oy + iz * oz) / std::max(inn * on, kEpsilon);
                c = std::max(-1.0, std::min(1.0, c));
                theta[in * NA + out] = std::abs(std::acos(c) * 180.0 / kPi);
            }
        }
    });
    std::vector<double> jac(NA);
    for (int in = 0; in < NA; ++in) {
        const double iy = t.omega[2 * in], iz = t.omega[2 * in + 1];
        jac[in] = std::pow(1.0 + iy * iy + iz * iz, -1.5);
    }
    // distinct theta values (all finite and >= +0, so == separates bit patterns)
    // (one sort of (value, position) pairs, then ranks in one pass)
    std::vector<std::pair<double, uint32_t>> order(NA2);
    for (size_t i = 0; i < NA2; ++i) order[i] = {theta[i], static_cast<uint32_t>(i)};
    std::sort(order.begin(), order.end());
    std::vector<double> uniq;
    std::vector<uint32_t> idx(NA2);
    for (size_t i = 0; i < NA2; ++i) {
        if (uniq.empty() || order[i].first != uniq.back()) uniq.push_back(order[i].first);
        idx[order[i].second] = static_cast<uint32_t>(uniq.size() - 1);
    }
    const size_t U = uniq.size();
    // uninitialised: every group's block is written below, in double or, for
    // a float-state context, as the float rounding of the same double values
    if (as_float) t.ker_v_f.resize(static_cast<size_t>(Ng) * NA2);
    else t.ker_v.resize(static_cast<size_t>(Ng) * NA2);
    auto group = [&](int ek, std::vector<double>& f, std::vector<double>& col) {
        double* K = as_float ? nullptr : t.ker_v.data() + static_cast<size_t>(ek) * NA2;
        float* Kf = as_float ? t.ker_v_f.data() + static_cast<size_t>(ek) * NA2 : nullptr;
        const double m1 = t.mu[ek * 3], m2 = t.mu[ek * 3 + 1];
        if (ek == Ng - 1 || m1 == 0.0 || m2 == 0.0) {
            if (as_float) std::fill(Kf, Kf + NA2, 0.0f);
            else std::fill(K, K + NA2, 0.0);
            return;
        }
        for (size_t u = 0; u < U; ++u) f[u] = std::pow(uniq[u], m1 - 1.0) * std::exp(-uniq[u] / m2);
        // column sums first, then each entry written once, already normalised
        std::fill(col.begin(), col.end(), 0.0);
        for (int in = 0; in < NA; ++in) {
            const double j = jac[in];
            const uint32_t* ir = idx.data() + static_cast<size_t>(in) * NA;
            for (int out = 0; out < NA; ++out) {
                const double v = f[ir[out]] * j;
                col[out] += std::isfinite(v) ? v : 0.0;
            }
        }
        for (int in = 0; in < NA; ++in) {
            const double j = jac[in];
            const uint32_t* ir = idx.data() + static_cast<size_t>(in) * NA;
            const size_t row = static_cast<size_t>(in) * NA;
            for (int out = 0; out < NA; ++out) {
                double v = f[ir[out]] * j;
                if (!std::isfinite(v)) v = 0.0;
                if (col[out] > kEpsilon) {
                    v /= col[out];
                    if (v < kKernelThreshold) v = 0.0;
                }
                if (as_float) Kf[row + out] = static_cast<float>(v);
                else K[row + out] = v;
            }
        }
    };
    const int n_threads = static_cast<int>(std::max(1u, std::min(32u, std::thread::hardware_concurrency())));
    const long long work = static_cast<long long>(Ng) * NA * NA;
    if (n_threads == 1 || work < (1 << 20)) {
        std::vector<double> f(U), col(NA);
        for (int ek = 0; ek < Ng; ++ek) group(ek, f, col);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    for (int i = 0; i < n_threads; ++i)
        pool.emplace_back([&] {
            std::vector<double> f(U), col(NA);
            for (int ek = next++; ek < Ng; ek = next++) group(ek, f, col);
        });
    for (auto& th : pool) th.join();
}

// Initial beam factors (initializeDistribution, bfpm_solver.cu:1815-2000).
bool beam_factors(const bfpn_grid& g, const bfpn_phys& p, BeamTables& t, std::string& err) {
    const Deltas& d = t.d;
    double cy = std::numeric_limits<double>::max(), cz = std::numeric_limits<double>::max();
    for (int j = 0; j < t.Nmu; ++j) cy = std::min(cy, std::abs(-0.5 * g.Lv + (j + 1) * d.dv));
    for (int i = 0; i < t.Nom; ++i) cz = std::min(cz, std::abs(-0.5 * g.Lu + (i + 1) * d.du));
    t.omega_center_y = cy;
    t.omega_center_z = cz;
    int ny_c = 0, nz_c = 0;
    double angular = 0.0;
    for (int j = 0; j < t.Nmu; ++j) {
        const double dy_ = std::abs(-0.5 * g.Lv + (j + 1) * d.dv) - cy;
        if (std::abs(dy_) < 0.25 * d.dv) ++ny_c;
        for (int i = 0; i < t.Nom; ++i) {
            const double dz_ = std::abs(-0.5 * g.Lu + (i + 1) * d.du) - cz;
            angular += std::exp(-p.a_2 * (dy_ * dy_ + dz_ * dz_)) * d.du * d.dv;
        }
    }
    for (int i = 0; i < t.Nom; ++i)
        if (std::abs(std::abs(-0.5 * g.Lu + (i + 1) * d.du) - cz) < 0.25 * d.du) ++nz_c;
    const bool discrete = p.flags & BFPN_FLAG_DISCRETE_ANGLE_DELTA;
    const bool trap = p.flags & BFPN_FLAG_TRAPEZOIDAL_YZ;
    if (discrete) angular = 1.0;
    double spatial = 0.0;
    for (int j = 0; j <= g.Nz; ++j) {
        const double z = -0.5 * g.Lz + j * d.dz;
        const double wz = trap && (j == 0 || j == g.Nz) ? 0.5 : 1.0;
        for (int i = 0; i <= g.Ny; ++i) {
            const double y = -0.5 * g.Ly + i * d.dy;
            const double wy = trap && (i == 0 || i == g.Ny) ? 0.5 : 1.0;
            spatial += wy * wz * std::exp(-p.a_1 * (y * y + z * z));
        }
    }
    spatial *= d.dy * d.dz;
    t.beam_e.resize(t.Ng);
    double energy = 0.0;
    for (int ek = 0; ek < t.Ng; ++ek) {
        const double E = (ek + 0.5) * d.dg + 1.0;
        t.beam_e[ek] = 1.0 / std::sqrt(2.0 * kPi) / p.sig_E
                       * std::exp(-std::pow((E - p.beam_energy) / p.sig_E / std::sqrt(2.0), 2));
        energy += t.beam_e[ek];
    }
    energy *= d.dg;
    const double mass = spatial * angular * energy;
    t.spatial_mass = spatial;
    t.angular_mass = angular;
    t.energy_mass = energy;
    if (!(mass > 0.0) || !std::isfinite(mass)) {
        err = "Initial beam has invalid discrete phase-space mass";
        return false;
    }
    const double scale = (p.flags & BFPN_FLAG_NORMALIZE_INITIAL_MASS) ? 1.0 / mass : 1.0;
    t.initial_scale = scale;
    t.beam_yza.assign(static_cast<size_t>(t.nyz) * t.NA, 0.0);
    for (int k = 0; k < t.NA; ++k) {
        const double d1 = std::abs(t.omega[2 * k]) - cy;
        const double d2 = std::abs(t.omega[2 * k + 1]) - cz;
        double ang = std::exp(-p.a_2 * (d1 * d1 + d2 * d2));
        if (discrete)
            ang = (std::abs(d1) < 0.25 * d.dv && std::abs(d2) < 0.25 * d.du) ? 1.0 / (ny_c * nz_c * d.du * d.dv) : 0.0;
        for (int j = 0; j <= g.Nz; ++j)
            for (int i = 0; i <= g.Ny; ++i) {
                const double y = -0.5 * g.Ly + i * d.dy;
                const double z = -0.5 * g.Lz + j * d.dz;
                t.beam_yza[static_cast<size_t>(j * (g.Ny + 1) + i) * t.NA + k] =
                    scale * std::exp(-p.a_1 * (y * y + z * z)) * ang;
            }
    }
    return true;
}

}  // namespace

void parallel_ranges(size_t n, size_t min_per_thread, const std::function<void(size_t, size_t)>& f) {
    const size_t hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const size_t nt = std::min(hw, std::max<size_t>(1, n / std::max<size_t>(1, min_per_thread)));
    if (nt <= 1) {
        f(0, n);
        return;
    }
    const size_t per = (n + nt - 1) / nt;
    std::vector<std::thread> pool;
    for (size_t i = 0; i < nt; ++i) {
        const size_t b = i * per, e = std::min(n, b + per);
        if (b < e) pool.emplace_back(f, b, e);
    }
    for (auto& th : pool) th.join();
}

const HostTable& angular_kernel_f64(BeamTables& t) {
    if (t.ker_v.empty() && t.Ng > 0 && t.NA > 0) angular_kernel(t, false);
    return t.ker_v;
}

Deltas compute_deltas(const bfpn_grid& g) {
    Deltas d;
    d.dt = g.Lx / g.Nx;
    d.dy = g.Ly / g.Ny;
    d.dz = g.Lz / g.Nz;
    d.dg = g.Lg / g.Ng;
    d.du = g.Lu / (g.Nom + 1);
    d.dv = g.Lv / (g.Nmu + 1);
    return d;
}

bool build_tables(const bfpn_grid& g, const bfpn_phys& p, const double* mu, int mu_rows, const double* sigma,
                  int sigma_rows, BeamTables& t, std::string& err, bool float_kernel) {
    t.Ng = g.Ng;
    t.Ny = g.Ny;
    t.Nz = g.Nz;
    t.Nmu = g.Nmu;
    t.Nom = g.Nom;
    t.nyz = (g.Ny + 1) * (g.Nz + 1);
    t.NA = g.Nmu * g.Nom;
    t.d = compute_deltas(g);
    const int Ng = g.Ng;
    if (mu_rows < Ng - 1) {
        err = "Scattering data has only " + std::to_string(mu_rows) + " rows; need at least " + std::to_string(Ng - 1);
        return false;
    }
    if (sigma_rows != Ng) {
        err = "Total cross-section data has " + std::to_string(sigma_rows) + " rows; need " + std::to_string(Ng);
        return false;
    }
    t.mu_rows = std::min(mu_rows, Ng);
    t.mu.assign(static_cast<size_t>(Ng) * 3, 0.0);
    std::copy(mu, mu + static_cast<size_t>(t.mu_rows) * 3, t.mu.begin());
    t.sigma.assign(sigma, sigma + Ng);
    if (p.flags & BFPN_FLAG_CALIBRATE_CROSS_SECTIONS) {  // bfpm_solver.cu:1487-1492
        for (double& s : t.sigma) s *= 0.9;
        for (int i = 401; i < 444 && i < Ng; ++i) t.sigma[i] -= 0.0002 * (0.5 + 0.5 * (i - 401));
    }
    t.en.resize(Ng + 1);
    for (int i = 0; i <= Ng; ++i) t.en[i] = i * t.d.dg + 1.0;
    // directions: omega_y runs over -v reversed, omega_z over -u (bfpm_solver.cu:1517-1531)
    t.omega.resize(2 * static_cast<size_t>(t.NA));
    for (int j = 0; j < t.Nmu; ++j)
        for (int i = 0; i < t.Nom; ++i) {
            const double v = -0.5 * g.Lv + (t.Nmu - j) * t.d.dv;  // v[Nmu-1-j]
            const double u = -0.5 * g.Lu + (i + 1) * t.d.du;
            t.omega[2 * (j * t.Nom + i)] = -v;
            t.omega[2 * (j * t.Nom + i) + 1] = -u;
        }
    stopping_power(g, p.material, t.d.dg, t.S_s);
    straggling(Ng, t.T_c);
    transport_cross_section(Ng, t.d.dg, t.sig_trg);
    energy_kernels(t);
    angular_kernel(t, float_kernel);
    t.sine_u.resize(static_cast<size_t>(t.Nom) * t.Nom);
    t.sine_v.resize(static_cast<size_t>(t.Nmu) * t.Nmu);
    for (int m = 0; m < t.Nom; ++m)
        for (int i = 0; i < t.Nom; ++i) t.sine_u[m * t.Nom + i] = std::sin(kPi * (m + 1) * (i + 1) / (t.Nom + 1));
    for (int m = 0; m < t.Nmu; ++m)
        for (int j = 0; j < t.Nmu; ++j) t.sine_v[m * t.Nmu + j] = std::sin(kPi * (m + 1) * (j + 1) / (t.Nmu + 1));
    return beam_factors(g, p, t, err);
}

std::vector<double> energy_coefficients(const BeamTables& t, const bfpn_phys& p, double dt) {
    const int Ng = t.Ng;
    const double rho = p.energy_density, dg = t.d.dg, idt = 1.0 / dt;
    const double dg2 = std::max(dg * dg, kEpsilon);
    const bool strag = p.flags & BFPN_FLAG_EQ15_STRAGGLING;
    std::vector<double> c(static_cast<size_t>(Ng) * kEnergyCoef, 0.0);
    for (int ek = 0; ek < Ng; ++ek) {
        double* k = c.data() + static_cast<size_t>(ek) * kEnergyCoef;
        const double sig = std::max(t.sigma[ek], 0.0);
        const double S_lo = std::max(t.S_s[ek], 0.0), S_hi = std::max(t.S_s[ek + 1], 0.0);
        const double a_lo = rho * S_lo / dg, a_hi = rho * S_hi / dg;
        const double inv_F = 1.0 / std::max(idt + 0.5 * a_lo + 0.5 * sig, kEpsilon);
        const double A = 1.5 * a_hi * inv_F;
        k[EC_INV_F] = inv_F;
        k[EC_A] = A;
        k[EC_F_FROM_F] = 0.5 * a_lo * inv_F;
        k[EC_F_FROM_HI] = 0.5 * a_hi * inv_F;
        k[EC_C_UP] = 0.5 * a_hi;
        k[EC_C_CUR] = -0.5 * a_lo;
        k[EC_C_F] = idt - 0.5 * sig;
        k[EC_R_F] = idt - 0.5 * sig - 0.5 * (a_hi - a_lo);
        k[EC_R_UP] = 1.5 * a_hi;
        k[EC_R_CUR] = 1.5 * a_lo;
        k[EC_R_FG] = -1.5 * (a_lo + a_hi);
        k[EC_R_HI] = 1.5 * a_hi - A * 0.5 * a_hi;
        const double coe = idt + 0.5 * sig + 1.5 * a_lo + 0.5 * (a_hi - a_lo) + A * 0.5 * a_lo;
        k[EC_INV_COE] = 1.0 / std::max(coe, kEpsilon);
        const double T_g = strag ? std::max(t.T_c[ek], 0.0) : 0.0;
        const double T_hi = (strag && ek + 1 < Ng) ? std::max(t.T_c[ek + 1], 0.0) : 0.0;
        const double T_lo = (strag && ek > 0) ? std::max(t.T_c[ek - 1], 0.0) : 0.0;
        k[EC_S_HI] = 0.5 * rho * T_hi / dg2;
        k[EC_S_LO] = 0.5 * rho * T_lo / dg2;
        k[EC_S_G] = rho * T_g / dg2;
        k[EC_L_IDT] = idt;
        k[EC_L_HI] = a_hi;
        k[EC_L_INV_DEN] = 1.0 / std::max(idt + a_lo + sig, kEpsilon);
        k[EC_L_LAP] = T_g > 0.0 ? 0.5 * dt * T_g / dg2 : 0.0;
    }
    return c;
}

std::vector<double> dose_coefficients(const BeamTables& t, const bfpn_phys& p) {
    const bool cat = p.flags & BFPN_FLAG_DOSE_CATASTROPHIC_LOSS;
    const double dg = t.d.dg;
    std::vector<double> c(2 * static_cast<size_t>(t.Ng));
    for (int ek = 0; ek < t.Ng; ++ek) {
        double w1 = 0.5 * (t.S_s[ek] + t.S_s[ek + 1]) * dg;
        double w2 = (t.S_s[ek + 1] - t.S_s[ek]) / 6.0 * dg;
        if (cat) {
            const double sig = std::max(t.sigma[ek], 0.0);
            w1 += 0.5 * (t.en[ek] + t.en[ek + 1]) * sig * dg;
            w2 += (t.en[ek + 1] - t.en[ek]) * sig * dg / 6.0;
        }
        c[2 * ek] = w1 / p.density;
        c[2 * ek + 1] = w2 / p.density;
    }
    return c;
}

std::vector<double> lite_coefficients(const BeamTables& t, double dt) {
    const double dg = t.d.dg;
    std::vector<double> c(2 * static_cast<size_t>(t.Ng));
    for (int ek = 0; ek < t.Ng; ++ek) {
        const double sig = std::max(t.sigma[ek], 0.0);
        const double S_lo = std::max(t.S_s[ek], 0.0), S_hi = std::max(t.S_s[ek + 1], 0.0);
        const double denom = 1.0 / dt + S_lo / dg + sig;
        c[2 * ek] = S_hi / dg;
        c[2 * ek + 1] = std::max(denom, kEpsilon);
    }
    return c;
}

std::vector<double> angle_factor(const BeamTables& t, const bfpn_phys& p, double dt) {
    const int Nom = t.Nom, Nmu = t.Nmu, NA = t.NA;
    const double norm = 4.0 / ((Nom + 1.0) * (Nmu + 1.0));
    std::vector<double> lu(Nom), lv(Nmu);
    for (int i = 0; i < Nom; ++i) lu[i] = (2.0 - 2.0 * std::cos(kPi * (i + 1) / (Nom + 1))) / (t.d.du * t.d.du);
    for (int j = 0; j < Nmu; ++j) lv[j] = (2.0 - 2.0 * std::cos(kPi * (j + 1) / (Nmu + 1))) / (t.d.dv * t.d.dv);
    std::vector<double> f(static_cast<size_t>(t.Ng) * NA);
    for (int ek = 0; ek < t.Ng; ++ek) {
        const double D = 0.5 * p.density * t.sig_trg[ek];
        for (int m = 0; m < NA; ++m) {
            const double lambda = D * (lu[m % Nom] + lv[m / Nom]);
            f[static_cast<size_t>(ek) * NA + m] = (2.0 / dt - lambda) / (2.0 / dt + lambda) * norm;
        }
    }
    return f;
}

bool read_table_files(const std::string& data_path, int Ng, std::vector<double>& mu, int& mu_rows,
                      std::vector<double>& sigma, int& sigma_rows, std::string& mu_path, std::string& err) {
    mu_path = data_path + "/data_cross.txt";
    std::ifstream mf(mu_path);
    if (!mf) {
        const size_t slash = data_path.find_last_of("/\\");
        const std::string material = data_path.substr(slash == std::string::npos ? 0 : slash + 1);
        if (material == "bone" || material == "air") {
            mu_path = data_path + "/data_" + material.substr(0, 1) + ".txt";
            mf.clear();
            mf.open(mu_path);
        }
    }
    if (!mf) {
        err = "Cannot open scattering data file in " + data_path;
        return false;
    }
    mu.assign(static_cast<size_t>(Ng) * 3, 0.0);
    mu_rows = 0;
    while (mu_rows < Ng && (mf >> mu[mu_rows * 3] >> mu[mu_rows * 3 + 1] >> mu[mu_rows * 3 + 2])) ++mu_rows;
    const std::string sigma_path = data_path + "/cross_total.txt";
    std::ifstream sf(sigma_path);
    if (!sf) {
        err = "Cannot open total cross-section file " + sigma_path;
        return false;
    }
    sigma.assign(Ng, 0.0);
    sigma_rows = 0;
    while (sigma_rows < Ng && (sf >> sigma[sigma_rows])) ++sigma_rows;
    return true;
}

}  // namespace bfpn
