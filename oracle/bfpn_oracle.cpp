// ORACLE -- test infrastructure only.
//
// CPU FP64 restatement of the reference's in-memory eq15 depth-step path
// (xiaojin1423764/BFPn_GPU).  It is the checker for the CUDA solver: only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
// load it.  The product never links or calls it.
//
// Parity is pinned against the reference's own golden IDD files
// (results/stage6_final_water230/{8_7,12_9}_nx1000/idd_output.txt); see the
// golden tests.  Every function cites the reference lines it restates.
//
// Build: oracle/Makefile  ->  oracle/liboracle.so (g++ -O2, no FMA contraction,
// so set-up tables are bit-identical to the reference's host code).

#include "../include/bfpn_capi.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// include/config.hpp:8-44
constexpr double PI = 3.14159265358979323846;
constexpr double ME = 9.10956e-31;
constexpr double MP = 1.673e-27;
constexpr double ALPHA = 1.0 / 137.0;
constexpr double C_LIGHT = 2.998e8;
constexpr double HBARC = 197.3;
constexpr double MEV_TO_J = 1.6e-13;
constexpr double EPSILON = 1e-10;
constexpr double KERNEL_THRESHOLD = 1e-3;
constexpr double SPARSE_THRESHOLD = 1e-5;

struct Elem { int Z; double w; };

// bfpm_solver.cu:150-154
static double mean_excitation_ev(int Z) {
    if (Z == 1) return 19.0;
    if (Z <= 13) return 11.2 + 11.7 * Z;
    return 52.8 + 8.71 * Z;
}

// bfpm_solver.cu:156-170
static double atomic_mass(int Z) {
    switch (Z) {
        case 1: return 1.0;
        case 6: return 12.0;
        case 7: return 14.0;
        case 8: return 16.0;
        case 11: return 23.0;
        case 12: return 24.0;
        case 15: return 31.0;
        case 16: return 32.0;
        case 18: return 40.0;
        case 20: return 40.0;
        default: return 2.0 * Z;
    }
}

// bfpm_solver.cu:172-182
static double bethe_element(double E, int Z) {
    const double kappa = 0.307;
    const double me_c2 = 0.51099895e6;
    double beta2 = E * (E + 2.0 * 938.3) / ((E + 938.3) * (E + 938.3));
    beta2 = std::max(beta2, EPSILON);
    double gamma2 = 1.0 / std::max(1.0 - beta2, EPSILON);
    double I = mean_excitation_ev(Z);
    double log_arg = std::max(2.0 * me_c2 * beta2 * gamma2 / I, 1.0 + EPSILON);
    double bracket = std::log(log_arg) - beta2;
    return kappa * (static_cast<double>(Z) / atomic_mass(Z)) / beta2 * bracket;
}

// bfpm_solver.cu:184-196 (mass fractions of the three presets)
static std::vector<Elem> composition(int material) {
    if (material == BFPN_MATERIAL_BONE)
        return {{1, 0.04200}, {6, 0.1940}, {7, 0.04000}, {8, 0.4250}, {11, 0.001000},
                {12, 0.002000}, {15, 0.09200}, {16, 0.003000}, {20, 0.2010}};
    if (material == BFPN_MATERIAL_AIR)
        return {{6, 0.0001248}, {7, 0.7553}, {8, 0.2318}, {18, 0.01283}};
    return {{1, 0.1111}, {8, 0.8889}};
}

struct Model {
    bfpn_grid g{};
    bfpn_phys p{};
    double dt = 0, dy = 0, dz = 0, dg = 0, du = 0, dv = 0;
    int Ng = 0, Ny = 0, Nz = 0, Nmu = 0, Nom = 0, nyz = 0, NA = 0;
    size_t per_e = 0, cells = 0;

    std::vector<double> mu, sigma, S_s, T_c, sig_trg, en, Omend;
    std::vector<double> ker_e1, ker_e2, ker_v, sine_u, sine_v;
    std::vector<int> beg, end;
    // non-zero entries of ker_v per (source group, input direction), outputs ascending
    std::vector<size_t> kv_ptr;
    std::vector<int> kv_out;
    std::vector<double> kv_w;
    std::vector<double> beam_yza, beam_e;
    std::vector<double> st[2][2];  // [species][coef]
    std::vector<double> source;
    std::vector<double> a1, a2;     // factorised source work arrays
    int steps_done = 0;
    bool direct_source = false;
    std::string err;

    size_t idx(int ek, int pos, int ang) const {
        return (static_cast<size_t>(ek) * nyz + pos) * NA + ang;
    }
};

// GridParams::computeDeltas, bfpm_solver.cu:1116-1127
static void compute_deltas(Model& m) {
    m.dt = m.g.Lx / m.g.Nx;
    m.dy = m.g.Ly / m.g.Ny;
    m.dz = m.g.Lz / m.g.Nz;
    m.dg = m.g.Lg / m.g.Ng;
    m.du = m.g.Lu / (m.g.Nom + 1);
    m.dv = m.g.Lv / (m.g.Nmu + 1);
}

// BFPnSolver::initialize table part, bfpm_solver.cu:1435-1568, and the
// physics-quantity builders 1570-1636.
static bool build_tables(Model& m, const double* mu_in, int mu_rows,
                         const double* sig_in, int sig_rows) {
    const int Ng = m.Ng;
    if (mu_rows < Ng - 1) { m.err = "scattering data has too few rows"; return false; }
    if (sig_rows != Ng) { m.err = "total cross-section data row count != Ng"; return false; }
    m.mu.assign(static_cast<size_t>(Ng) * 3, 0.0);
    for (int r = 0; r < std::min(mu_rows, Ng); ++r)
        for (int c = 0; c < 3; ++c) m.mu[r * 3 + c] = mu_in[r * 3 + c];
    m.sigma.assign(sig_in, sig_in + Ng);
    if (m.p.flags & BFPN_FLAG_CALIBRATE_CROSS_SECTIONS) {  // bfpm_solver.cu:1487-1492
        for (auto& s : m.sigma) s *= 0.9;
        for (int i = 401; i < 444 && i < Ng; i++) m.sigma[i] -= 0.0002 * (0.5 + 0.5 * (i - 401));
    }

    m.en.resize(Ng + 1);
    for (int i = 0; i <= Ng; i++) m.en[i] = i * m.dg + 1.0;  // :1510

    // directions, bfpm_solver.cu:1517-1531
    const int NA = m.NA;
    std::vector<double> u(m.Nom), v(m.Nmu);
    for (int i = 0; i < m.Nom; i++) u[i] = -0.5 * m.g.Lu + (i + 1) * m.du;
    for (int j = 0; j < m.Nmu; j++) v[j] = -0.5 * m.g.Lv + (j + 1) * m.dv;
    m.Omend.resize(static_cast<size_t>(NA) * 2);
    for (int j = 0; j < m.Nmu; j++)
        for (int i = 0; i < m.Nom; i++) {
            int id = j * m.Nom + i;
            m.Omend[id * 2] = -v[m.Nmu - 1 - j];
            m.Omend[id * 2 + 1] = -u[i];
        }

    // computeStoppingPower, bfpm_solver.cu:1570-1597
    const auto comp = composition(m.p.material);
    const auto water = composition(BFPN_MATERIAL_WATER);
    m.S_s.resize(Ng + 1);
    for (int i = 0; i <= Ng; i++) {
        double E = (i == 0) ? 1.0 : (i == Ng) ? m.g.Lg + 1.0 : (i - 0.5) * m.dg + 1.0;
        double weighted = 0.0;
        for (const auto& e : comp) weighted += e.w * bethe_element(E, e.Z);
        double ww = 0.0;
        for (const auto& e : water) ww += e.w * bethe_element(E, e.Z);
        double beta_2 = E * (E + 2.0 * 938.3) / std::pow(E + 938.3, 2);
        double F_beta = std::log(1.02e6 * beta_2 / (1.0 - beta_2)) - beta_2 - 4.31;
        double water_legacy = 0.170 / beta_2 * F_beta + 0.02;
        double scale = (ww > EPSILON) ? weighted / ww : 1.0;
        m.S_s[i] = water_legacy * scale;
    }

    // computeStraggling, bfpm_solver.cu:1599-1615 (a constant)
    m.T_c.resize(Ng);
    for (int i = 0; i < Ng; i++) {
        double eta = 8.99e18 * 4.0 * PI * std::pow(1.6e-19, 4) / std::pow(1.6e-13, 2) / 100.0;
        m.T_c[i] = eta * 3.34e29 * 1.2;
    }

    // computeTransportCrossSection, bfpm_solver.cu:1617-1636
    m.sig_trg.resize(Ng);
    for (int i = 0; i < Ng; i++) {
        double E = (i + 0.5) * m.dg + 1.0;
        double vel = std::sqrt(2.0 * E * MEV_TO_J / MP);
        double beta = vel / (3.0 * C_LIGHT);
        double Zt = 3;
        double eta = std::pow(Zt, 2.0 / 3.0) * std::pow(ALPHA, 2) * std::pow(ME / MP, 2) / (beta * beta);
        double mid = std::log((eta + 1.0) / eta) - 1.0 / (eta + 1.0);
        m.sig_trg[i] = 2.0 * PI * 3.34 * std::pow(HBARC, 2) * std::pow(ALPHA, 2) / 4.0 * Zt * Zt
                       / (E * E) * mid / 1000.0;
    }

    // initializeKernels, bfpm_solver.cu:1638-1700: ker_e, ker_e1, ker_e2
    const size_t NN = static_cast<size_t>(Ng) * Ng;
    std::vector<double> init(NN, 0.0), shifted(NN, 0.0), ker_e(NN, 0.0);
    for (int j = 0; j < Ng - 1; j++)
        for (int i = 0; i < Ng - 1; i++) {
            double mu3 = m.mu[j * 3 + 2];
            if (mu3 == 0) init[i * Ng + j] = 0.0;
            else if (i < j) init[i * Ng + j] = 0.0;
            else init[i * Ng + j] = m.dg / mu3 * std::exp(-(i - j + 0.5) * m.dg / mu3);
        }
    for (int j = 0; j < Ng - 1; ++j)
        for (int i = 0; i < Ng; ++i) {
            if (i == j) shifted[i * Ng + j] = 0.0;
            else if (i < j) shifted[i * Ng + j] = init[i * Ng + j];
            else shifted[i * Ng + j] = init[(i - 1) * Ng + j];
        }
    for (int row = 0; row < Ng; ++row)
        for (int col = 0; col < Ng; ++col) {
            double value = shifted[(Ng - 1 - row) * Ng + (Ng - 1 - col)];
            if (std::abs(value) < SPARSE_THRESHOLD) value = 0.0;
            ker_e[row * Ng + col] = value * m.sigma[col];
        }
    m.ker_e1.assign(NN, 0.0);
    m.ker_e2.assign(NN, 0.0);
    for (int row = 0; row < Ng; ++row)
        for (int col = 0; col < Ng; ++col) {
            double cur = ker_e[row * Ng + col];
            double next = (row + 1 < Ng) ? ker_e[(row + 1) * Ng + col] : 0.0;
            m.ker_e1[row * Ng + col] = 0.5 * (cur + next);
            m.ker_e2[row * Ng + col] = 0.5 * (-cur + next);
        }
    // band limits, bfpm_solver.cu:1702-1721
    m.beg.assign(Ng, Ng);
    m.end.assign(Ng, 0);
    for (int row = 0; row < Ng; ++row) {
        for (int col = 0; col < Ng; ++col) {
            if (m.ker_e1[row * Ng + col] != 0.0 || m.ker_e2[row * Ng + col] != 0.0) {
                m.beg[row] = std::min(m.beg[row], col);
                m.end[row] = std::max(m.end[row], col + 1);
            }
        }
        if (m.beg[row] == Ng) { m.beg[row] = 0; m.end[row] = 0; }
    }

    // angular kernel ker_v[src][in][out], bfpm_solver.cu:1723-1790
    std::vector<double> angles(static_cast<size_t>(NA) * NA, 0.0);
    for (int out = 0; out < NA; ++out) {
        double oy = m.Omend[out * 2], oz = m.Omend[out * 2 + 1];
        double on = std::sqrt(1.0 + oy * oy + oz * oz);
        for (int in = 0; in < NA; ++in) {
            double iy = m.Omend[in * 2], iz = m.Omend[in * 2 + 1];
            double inn = std::sqrt(1.0 + iy * iy + iz * iz);
            double c = (1.0 + iy * oy + iz * oz) / std::max(inn * on, EPSILON);
            c = std::max(-1.0, std::min(1.0, c));
            angles[static_cast<size_t>(in) * NA + out] = std::abs(std::acos(c) * 180.0 / PI);
        }
    }
    m.ker_v.assign(static_cast<size_t>(Ng) * NA * NA, 0.0);
    for (int ek = 0; ek < Ng - 1; ++ek) {
        if (m.mu[ek * 3 + 0] == 0.0 || m.mu[ek * 3 + 1] == 0.0) continue;
        for (int out = 0; out < NA; ++out) {
            double col_sum = 0.0;
            for (int in = 0; in < NA; ++in) {
                double theta = angles[static_cast<size_t>(in) * NA + out];
                double iy = m.Omend[in * 2], iz = m.Omend[in * 2 + 1];
                double value = std::pow(theta, m.mu[ek * 3 + 0] - 1.0) * std::exp(-theta / m.mu[ek * 3 + 1])
                               * std::pow(1.0 + iy * iy + iz * iz, -1.5);
                if (!std::isfinite(value)) value = 0.0;
                m.ker_v[(static_cast<size_t>(ek) * NA + in) * NA + out] = value;
                col_sum += value;
            }
            if (col_sum > EPSILON) {
                for (int in = 0; in < NA; ++in) {
                    double& value = m.ker_v[(static_cast<size_t>(ek) * NA + in) * NA + out];
                    value /= col_sum;
                    if (value < KERNEL_THRESHOLD) value = 0.0;
                }
            }
        }
    }

    m.kv_ptr.assign(static_cast<size_t>(Ng) * NA + 1, 0);
    m.kv_out.clear();
    m.kv_w.clear();
    for (size_t r = 0; r < static_cast<size_t>(Ng) * NA; ++r) {
        m.kv_ptr[r] = m.kv_w.size();
        for (int out = 0; out < NA; ++out) {
            double w = m.ker_v[r * NA + out];
            if (w != 0.0) {
                m.kv_out.push_back(out);
                m.kv_w.push_back(w);
            }
        }
    }
    m.kv_ptr[static_cast<size_t>(Ng) * NA] = m.kv_w.size();

    // sine tables, angle_diffusion.cu:381-413
    m.sine_u.resize(static_cast<size_t>(m.Nom) * m.Nom);
    m.sine_v.resize(static_cast<size_t>(m.Nmu) * m.Nmu);
    for (int a = 0; a < m.Nom; ++a)
        for (int i = 0; i < m.Nom; ++i)
            m.sine_u[static_cast<size_t>(a) * m.Nom + i] = std::sin(PI * (a + 1) * (i + 1) / (m.Nom + 1));
    for (int a = 0; a < m.Nmu; ++a)
        for (int j = 0; j < m.Nmu; ++j)
            m.sine_v[static_cast<size_t>(a) * m.Nmu + j] = std::sin(PI * (a + 1) * (j + 1) / (m.Nmu + 1));
    return true;
}

// initializeDistribution, full mode, bfpm_solver.cu:1815-2026.  The state is
// the product f1(pos, ang) * f2(ek), each factor evaluated exactly as there.
static bool init_beam(Model& m) {
    const int Nmu = m.Nmu, Nom = m.Nom;
    double c1 = std::numeric_limits<double>::max(), c2 = std::numeric_limits<double>::max();
    for (int j = 0; j < Nmu; ++j) c1 = std::min(c1, std::abs(-0.5 * m.g.Lv + (j + 1) * m.dv));
    for (int i = 0; i < Nom; ++i) c2 = std::min(c2, std::abs(-0.5 * m.g.Lu + (i + 1) * m.du));
    int n1 = 0, n2 = 0;
    double angular_mass = 0.0;
    for (int j = 0; j < Nmu; ++j) {
        double v = -0.5 * m.g.Lv + (j + 1) * m.dv;
        double delta = std::abs(v) - c1;
        if (std::abs(delta) < 0.25 * m.dv) ++n1;
        for (int i = 0; i < Nom; ++i) {
            double u = -0.5 * m.g.Lu + (i + 1) * m.du;
            double du_ = std::abs(u) - c2;
            angular_mass += std::exp(-m.p.a_2 * (delta * delta + du_ * du_)) * m.du * m.dv;
        }
    }
    for (int i = 0; i < Nom; ++i) {
        double u = -0.5 * m.g.Lu + (i + 1) * m.du;
        if (std::abs(std::abs(u) - c2) < 0.25 * m.du) ++n2;
    }
    const bool discrete = m.p.flags & BFPN_FLAG_DISCRETE_ANGLE_DELTA;
    const bool trap = m.p.flags & BFPN_FLAG_TRAPEZOIDAL_YZ;
    if (discrete) angular_mass = 1.0;
    double spatial_mass = 0.0;
    for (int j = 0; j <= m.Nz; ++j) {
        double z = -0.5 * m.g.Lz + j * m.dz;
        double wz = trap && (j == 0 || j == m.Nz) ? 0.5 : 1.0;
        for (int i = 0; i <= m.Ny; ++i) {
            double y = -0.5 * m.g.Ly + i * m.dy;
            double wy = trap && (i == 0 || i == m.Ny) ? 0.5 : 1.0;
            spatial_mass += wy * wz * std::exp(-m.p.a_1 * (y * y + z * z));
        }
    }
    spatial_mass *= m.dy * m.dz;
    double energy_mass = 0.0;
    for (int ek = 0; ek < m.Ng; ++ek) {
        double E = (ek + 0.5) * m.dg + 1.0;
        energy_mass += 1.0 / std::sqrt(2.0 * PI) / m.p.sig_E
                       * std::exp(-std::pow((E - m.p.beam_energy) / m.p.sig_E / std::sqrt(2.0), 2));
    }
    energy_mass *= m.dg;
    double mass = spatial_mass * angular_mass * energy_mass;
    if (!(mass > 0.0) || !std::isfinite(mass)) { m.err = "Initial beam has invalid discrete phase-space mass"; return false; }
    double scale = (m.p.flags & BFPN_FLAG_NORMALIZE_INITIAL_MASS) ? 1.0 / mass : 1.0;

    m.beam_yza.assign(static_cast<size_t>(m.nyz) * m.NA, 0.0);
    for (int k = 0; k < m.NA; k++) {
        double o1 = m.Omend[k * 2], o2 = m.Omend[k * 2 + 1];
        for (int j = 0; j <= m.Nz; j++)
            for (int i = 0; i <= m.Ny; i++) {
                double y = -0.5 * m.g.Ly + i * m.dy;
                double z = -0.5 * m.g.Lz + j * m.dz;
                double d1 = std::abs(o1) - c1;
                double d2 = std::abs(o2) - c2;
                double angular = std::exp(-m.p.a_2 * (d1 * d1 + d2 * d2));
                if (discrete) {
                    bool sel = std::abs(d1) < 0.25 * m.dv && std::abs(d2) < 0.25 * m.du;
                    angular = sel ? 1.0 / (n1 * n2 * m.du * m.dv) : 0.0;
                }
                m.beam_yza[static_cast<size_t>(j * (m.Ny + 1) + i) * m.NA + k] =
                    scale * std::exp(-m.p.a_1 * (y * y + z * z)) * angular;
            }
    }
    m.beam_e.resize(m.Ng);
    for (int ek = 0; ek < m.Ng; ek++) {
        double E = (ek + 0.5) * m.dg + 1.0;
        m.beam_e[ek] = 1.0 / std::sqrt(2.0 * PI) / m.p.sig_E
                       * std::exp(-std::pow((E - m.p.beam_energy) / m.p.sig_E / std::sqrt(2.0), 2));
    }
    for (int s = 0; s < 2; ++s)
        for (int c = 0; c < 2; ++c) m.st[s][c].assign(m.p.flags & BFPN_FLAG_LITE_MEMORY ? 0 : m.cells, 0.0);
    auto& F = m.st[0][0];
    if (m.p.flags & BFPN_FLAG_LITE_MEMORY) {
        // initializeLiteDistributionKernel, bfpm_solver.cu:993-1050:
        // F = initial_scale * f1 * f2 with f1 = exp(-a1 (y^2+z^2)) * angular
        F.assign(m.cells, 0.0);
#pragma omp parallel for schedule(static)
        for (int ek = 0; ek < m.Ng; ++ek)
            for (int j = 0; j <= m.Nz; ++j)
                for (int i = 0; i <= m.Ny; ++i)
                    for (int k = 0; k < m.NA; ++k) {
                        double y = -0.5 * m.g.Ly + i * m.dy;
                        double z = -0.5 * m.g.Lz + j * m.dz;
                        double d1 = std::abs(m.Omend[2 * k]) - c1;
                        double d2 = std::abs(m.Omend[2 * k + 1]) - c2;
                        double angular = std::exp(-m.p.a_2 * (d1 * d1 + d2 * d2));
                        if (discrete) {
                            bool sel = std::abs(d1) < 0.25 * m.dv && std::abs(d2) < 0.25 * m.du;
                            angular = sel ? 1.0 / (n1 * n2 * m.du * m.dv) : 0.0;
                        }
                        double f1 = std::exp(-m.p.a_1 * (y * y + z * z)) * angular;
                        double E = (ek + 0.5) * m.dg + 1.0;
                        double f2 = 1.0 / std::sqrt(2.0 * PI) / m.p.sig_E *
                                    std::exp(-std::pow((E - m.p.beam_energy) / m.p.sig_E / std::sqrt(2.0), 2));
                        F[m.idx(ek, j * (m.Ny + 1) + i, k)] = scale * f1 * f2;
                    }
        m.steps_done = 0;
        return true;
    }
#pragma omp parallel for schedule(static)
    for (int ek = 0; ek < m.Ng; ++ek)
        for (size_t l = 0; l < m.per_e; ++l) F[ek * m.per_e + l] = m.beam_yza[l] * m.beam_e[ek];
    m.steps_done = 0;
    return true;
}

// energyDgCnKernel, energy_solver.cu:41-161 (eq15 branch 108-159, legacy
// branch 88-106), applied in place as EnergyDepositionSolver::solve does
// (new values into temporaries, then copied back, energy_solver.cu:444-506).
static void energy_sweep(Model& m, int species, double dt, const double* source) {
    const int Ng = m.Ng;
    const size_t per_e = m.per_e;
    const double density = m.p.energy_density;
    const double dg = m.dg;
    const bool legacy = m.p.flags & BFPN_FLAG_LEGACY_ENERGY;
    const bool strag = m.p.flags & BFPN_FLAG_EQ15_STRAGGLING;
    double* Fa = m.st[species][0].data();
    double* fa = m.st[species][1].data();
    const double dg2 = std::max(dg * dg, EPSILON);
#pragma omp parallel
    {
        std::vector<double> Fo(Ng), fo(Ng);
#pragma omp for schedule(static)
        for (long long lane = 0; lane < static_cast<long long>(per_e); ++lane) {
            for (int ek = 0; ek < Ng; ++ek) {
                Fo[ek] = Fa[ek * per_e + lane];
                fo[ek] = fa[ek * per_e + lane];
            }
            auto ldF = [&](int ek) { return (ek < 0 || ek >= Ng) ? 0.0 : Fo[ek]; };
            auto ldf = [&](int ek) { return (ek < 0 || ek >= Ng) ? 0.0 : fo[ek]; };
            double next_F = 0.0, next_f = 0.0;
            for (int ek = Ng - 1; ek >= 0; --ek) {
                const size_t id = ek * per_e + lane;
                double Fg = Fo[ek];
                double fg = fo[ek];
                double sig = std::max(m.sigma[ek], 0.0);
                double S_lo = std::max(m.S_s[ek], 0.0);
                double S_hi = std::max(m.S_s[ek + 1], 0.0);
                double src = source ? source[id] : 0.0;
                double T_g = strag ? std::max(m.T_c[ek], 0.0) : 0.0;
                double T_hi = (strag && ek + 1 < Ng) ? std::max(m.T_c[ek + 1], 0.0) : 0.0;
                double T_lo = (strag && ek > 0) ? std::max(m.T_c[ek - 1], 0.0) : 0.0;
                if (legacy) {
                    double denom = 1.0 / dt + density * S_lo / dg + sig;
                    double F_val = (std::max(Fg, 0.0) / dt + density * S_hi / dg * next_F + src)
                                   / std::max(denom, EPSILON);
                    double f_val = (fg / dt + density * S_hi / dg * next_f) / std::max(denom, EPSILON);
                    if (T_g > 0.0) {
                        double lap = std::max(ldF(ek + 1), 0.0) - 2.0 * std::max(Fg, 0.0)
                                     + std::max(ldF(ek - 1), 0.0);
                        F_val += 0.5 * dt * T_g / dg2 * lap;
                    }
                    Fa[id] = std::max(F_val, 0.0);
                    fa[id] = std::max(f_val, 0.0);
                    next_F = Fa[id];
                    next_f = fa[id];
                    continue;
                }
                const double p1_hi = ldF(ek + 1), p2_hi = ldf(ek + 1), p1_lo = ldF(ek - 1);
                const double up = p1_hi - p2_hi;
                const double cur = Fg - fg;
                const double den_F = std::max(1.0 / dt + 0.5 * density * S_lo / dg + 0.5 * sig, EPSILON);
                const double inv_F = 1.0 / den_F;
                const double A = (1.5 * density * S_hi / dg) * inv_F;
                const double F_from_f = (0.5 * density * S_lo / dg) * inv_F;
                const double F_from_hi = (0.5 * density * S_hi / dg) * inv_F;
                const double strag_rhs = 0.5 * density * T_hi / dg2 * p1_hi + 0.5 * density * T_lo / dg2 * p1_lo
                                         - density * T_g / dg2 * Fg;
                const double common = 0.5 * density * S_hi / dg * up - 0.5 * density * S_lo / dg * cur
                                      - 0.5 * sig * Fg + Fg / dt + strag_rhs + src;
                const double rhs4 = inv_F * common;
                const double rhs1e = fg / dt - 0.5 * sig * fg;
                const double rhs2e = 1.5 * density * S_hi / dg * up + 1.5 * density * S_lo / dg * cur
                                     - 1.5 * density * (S_lo + S_hi) / dg * Fg
                                     - 0.5 * density * (S_hi - S_lo) / dg * fg;
                const double rhs3e = A * common;
                const double high2 = 1.5 * density * S_hi / dg;
                const double hi_delta = next_F - next_f;
                const double rhs = rhs1e + rhs2e - rhs3e + (high2 - A * 0.5 * density * S_hi / dg) * hi_delta;
                const double coe = 1.0 / dt + 0.5 * sig + 1.5 * density * S_lo / dg
                                   + 0.5 * density * (S_hi - S_lo) / dg + A * 0.5 * density * S_lo / dg;
                double f_val = rhs / std::max(coe, EPSILON);
                double F_val = F_from_f * f_val + rhs4 + F_from_hi * hi_delta;
                Fa[id] = F_val;
                fa[id] = f_val;
                next_F = F_val;
                next_f = f_val;
            }
        }
    }
}

// muscl_paper_slope, spatial_transport.cu:23-29
static inline double slope(double l, double c, double r) {
    double fwd = r - c;
    if (std::fabs(fwd) < EPSILON) return 0.0;
    double theta = (c - l) / fwd;
    double eta = std::max(0.0, std::max(std::min(2.0 * theta, 1.0), std::min(theta, 2.0)));
    return fwd * eta;
}

// spatial_flux_divergence_value, spatial_transport.cu:31-102, for all
// (pos, ang) of one energy plane block X[pos][ang].
static void flux_div(const Model& m, const double* X, double* div) {
    const int Ny = m.Ny, Nz = m.Nz, NA = m.NA, Ny1 = m.Ny + 1;
    for (int j = 0; j <= Nz; ++j)
        for (int i = 0; i <= Ny; ++i) {
            const int s = j * Ny1 + i;
            const int im2 = std::max(0, i - 2), im1 = std::max(0, i - 1);
            const int ip1 = std::min(Ny, i + 1), ip2 = std::min(Ny, i + 2);
            const int jm2 = std::max(0, j - 2), jm1 = std::max(0, j - 1);
            const int jp1 = std::min(Nz, j + 1), jp2 = std::min(Nz, j + 2);
            for (int a = 0; a < NA; ++a) {
                const double wy = m.Omend[2 * a], wz = m.Omend[2 * a + 1];
                const double c = X[static_cast<size_t>(s) * NA + a];
                auto at = [&](int ii, int jj) { return X[static_cast<size_t>(jj * Ny1 + ii) * NA + a]; };
                double ym2 = at(im2, j), ym1 = at(im1, j), yp1 = at(ip1, j), yp2 = at(ip2, j);
                double sy_m1 = slope(ym2, ym1, c), sy_0 = slope(ym1, c, yp1), sy_p1 = slope(c, yp1, yp2);
                double lfy, rfy;
                if (wy >= 0.0) { lfy = wy * (ym1 + 0.5 * sy_m1); rfy = wy * (c + 0.5 * sy_0); }
                else { lfy = wy * (c - 0.5 * sy_0); rfy = wy * (yp1 - 0.5 * sy_p1); }
                double zm2 = at(i, jm2), zm1 = at(i, jm1), zp1 = at(i, jp1), zp2 = at(i, jp2);
                double sz_m1 = slope(zm2, zm1, c), sz_0 = slope(zm1, c, zp1), sz_p1 = slope(c, zp1, zp2);
                double lfz, rfz;
                if (wz >= 0.0) { lfz = wz * (zm1 + 0.5 * sz_m1); rfz = wz * (c + 0.5 * sz_0); }
                else { lfz = wz * (c - 0.5 * sz_0); rfz = wz * (zp1 - 0.5 * sz_p1); }
                div[static_cast<size_t>(s) * NA + a] = (rfy - lfy) / m.dy + (rfz - lfz) / m.dz;
            }
        }
}

// SpatialTransportSolver::solveEq18, spatial_transport.cu:134-161, 202-262:
// predictor p = F - dt*div(F), corrector F - dt/2*(div F + div p), each
// clipped at 0 unless preserve_sign.
static void transport(Model& m, int species, int coef, double dt, bool preserve_sign) {
    double* F = m.st[species][coef].data();
    const size_t per_e = m.per_e;
#pragma omp parallel
    {
        std::vector<double> d0(per_e), pred(per_e), d1(per_e);
#pragma omp for schedule(static)
        for (int ek = 0; ek < m.Ng; ++ek) {
            double* X = F + ek * per_e;
            flux_div(m, X, d0.data());
            for (size_t l = 0; l < per_e; ++l) {
                double v = X[l] - dt * d0[l];
                pred[l] = preserve_sign ? v : std::max(v, 0.0);
            }
            flux_div(m, pred.data(), d1.data());
            for (size_t l = 0; l < per_e; ++l) {
                double v = X[l] - 0.5 * dt * (d0[l] + d1[l]);
                X[l] = preserve_sign ? v : std::max(v, 0.0);
            }
        }
    }
}

// AngleDiffusionSolver::solveEq19, angle_diffusion.cu:420-483 with the factor
// of buildDiffusionFactorKernel (7-34) and complexToRealKernel (75-80), and
// the four separable DST-I passes (254-362), per (ek, pos) slice X[v][u].
static void angle(Model& m, int species, int coef, double dt) {
    const int Nom = m.Nom, Nmu = m.Nmu, NA = m.NA, Ng = m.Ng;
    std::vector<double> fac(static_cast<size_t>(Ng) * NA);
    const double norm = 4.0 / ((Nom + 1.0) * (Nmu + 1.0));
    for (int ek = 0; ek < Ng; ++ek)
        for (int id = 0; id < NA; ++id) {
            int i = id % Nom, j = id / Nom;
            double lu = (2.0 - 2.0 * std::cos(PI * (i + 1) / (Nom + 1))) / (m.du * m.du);
            double lv = (2.0 - 2.0 * std::cos(PI * (j + 1) / (Nmu + 1))) / (m.dv * m.dv);
            double D = 0.5 * m.p.density * m.sig_trg[ek];
            double lambda = D * (lu + lv);
            double ratio = (2.0 / dt - lambda) / (2.0 / dt + lambda);
            fac[static_cast<size_t>(ek) * NA + id] = ratio * norm;
        }
    double* F = m.st[species][coef].data();
    const long long slices = static_cast<long long>(Ng) * m.nyz;
#pragma omp parallel
    {
        std::vector<double> t1(NA), t2(NA);
#pragma omp for schedule(static)
        for (long long b = 0; b < slices; ++b) {
            double* X = F + b * NA;
            const int ek = static_cast<int>(b / m.nyz);
            for (int v = 0; v < Nmu; ++v)  // forward u
                for (int mu = 0; mu < Nom; ++mu) {
                    double s = 0.0;
                    for (int a = 0; a < Nom; ++a) s += X[v * Nom + a] * m.sine_u[mu * Nom + a];
                    t1[v * Nom + mu] = s;
                }
            for (int nu = 0; nu < Nmu; ++nu)  // forward v and factor
                for (int mu = 0; mu < Nom; ++mu) {
                    double s = 0.0;
                    for (int v = 0; v < Nmu; ++v) s += m.sine_v[nu * Nmu + v] * t1[v * Nom + mu];
                    t2[nu * Nom + mu] = s * fac[static_cast<size_t>(ek) * NA + nu * Nom + mu];
                }
            for (int v = 0; v < Nmu; ++v)  // inverse v
                for (int mu = 0; mu < Nom; ++mu) {
                    double s = 0.0;
                    for (int nu = 0; nu < Nmu; ++nu) s += m.sine_v[nu * Nmu + v] * t2[nu * Nom + mu];
                    t1[v * Nom + mu] = s;
                }
            for (int v = 0; v < Nmu; ++v)  // inverse u
                for (int a = 0; a < Nom; ++a) {
                    double s = 0.0;
                    for (int mu = 0; mu < Nom; ++mu) s += t1[v * Nom + mu] * m.sine_u[mu * Nom + a];
                    X[v * Nom + a] = s;
                }
        }
    }
}

// secondarySourceFromPrimaryKernel, energy_solver.cu:287-333, in the
// reference's own summation order (small cases; cross-checks the factorised
// form below).
static void source_direct(Model& m) {
    const int Ng = m.Ng, NA = m.NA, nyz = m.nyz;
    const double* P1 = m.st[0][0].data();
    const double* P2 = m.st[0][1].data();
    m.source.assign(m.cells, 0.0);
#pragma omp parallel for schedule(static)
    for (long long gid = 0; gid < static_cast<long long>(m.cells); ++gid) {
        int ek = static_cast<int>(gid / m.per_e);
        long long rem = gid - static_cast<long long>(ek) * m.per_e;
        int cell = static_cast<int>(rem / NA);
        int out = static_cast<int>(rem - static_cast<long long>(cell) * NA);
        double q1 = 0.0, q2 = 0.0;
        int sb = std::max(0, m.beg[ek]), se = std::min(Ng, m.end[ek]);
        for (int s = sb; s < se; ++s) {
            double e1 = m.ker_e1[static_cast<size_t>(ek) * Ng + s];
            double e2 = m.ker_e2[static_cast<size_t>(ek) * Ng + s];
            if (e1 == 0.0 && e2 == 0.0) continue;
            const double* kv = m.ker_v.data() + static_cast<size_t>(s) * NA * NA;
            for (int in = 0; in < NA; ++in) {
                double w = kv[static_cast<size_t>(in) * NA + out];
                if (w == 0.0) continue;
                size_t si = (static_cast<size_t>(s) * nyz + cell) * NA + in;
                q1 += std::max(P1[si], 0.0) * e1 * w;
                q2 += P2[si] * e2 * w;
            }
        }
        m.source[gid] = m.dg * (q1 + q2 / 3.0);
    }
}

// The same sum factorised: angular contraction per source group, then the
// banded energy contraction (FP64 reordering only).
static void source_factorised(Model& m) {
    const int Ng = m.Ng, NA = m.NA;
    const size_t per_e = m.per_e;
    const double* P1 = m.st[0][0].data();
    const double* P2 = m.st[0][1].data();
    m.a1.assign(m.cells, 0.0);
    m.a2.assign(m.cells, 0.0);
    std::vector<char> used(Ng, 0);
    for (int ek = 0; ek < Ng; ++ek)
        for (int s = std::max(0, m.beg[ek]); s < std::min(Ng, m.end[ek]); ++s) used[s] = 1;
#pragma omp parallel for schedule(dynamic, 4)
    for (long long b = 0; b < static_cast<long long>(Ng) * m.nyz; ++b) {
        int s = static_cast<int>(b / m.nyz);
        if (!used[s]) continue;
        const double* p1 = P1 + b * NA;
        const double* p2 = P2 + b * NA;
        double* o1 = m.a1.data() + b * NA;
        double* o2 = m.a2.data() + b * NA;
        // zero kernel entries are skipped (they add exact zeros), which keeps
        // the dense order of summation for every output
        for (int in = 0; in < NA; ++in) {
            double x1 = std::max(p1[in], 0.0), x2 = p2[in];
            const size_t r = static_cast<size_t>(s) * NA + in;
            for (size_t k = m.kv_ptr[r]; k < m.kv_ptr[r + 1]; ++k) {
                o1[m.kv_out[k]] += x1 * m.kv_w[k];
                o2[m.kv_out[k]] += x2 * m.kv_w[k];
            }
        }
    }
    m.source.assign(m.cells, 0.0);
#pragma omp parallel
    {
        std::vector<double> q1(per_e), q2(per_e);
#pragma omp for schedule(dynamic, 1)
        for (int ek = 0; ek < Ng; ++ek) {
            std::fill(q1.begin(), q1.end(), 0.0);
            std::fill(q2.begin(), q2.end(), 0.0);
            for (int s = std::max(0, m.beg[ek]); s < std::min(Ng, m.end[ek]); ++s) {
                double e1 = m.ker_e1[static_cast<size_t>(ek) * Ng + s];
                double e2 = m.ker_e2[static_cast<size_t>(ek) * Ng + s];
                const double* x1 = m.a1.data() + s * per_e;
                const double* x2 = m.a2.data() + s * per_e;
                for (size_t l = 0; l < per_e; ++l) {
                    q1[l] += e1 * x1[l];
                    q2[l] += e2 * x2[l];
                }
            }
            double* out = m.source.data() + ek * per_e;
            for (size_t l = 0; l < per_e; ++l) out[l] = m.dg * (q1[l] + q2[l] / 3.0);
        }
    }
}

static void secondary_source(Model& m) {
    if (m.direct_source) source_direct(m);
    else source_factorised(m);
}

// integratedDepthDoseKernel (bfpm_solver.cu:229-309) and
// computeScalarDoseProxy (3418-3444).
static void idd(const Model& m, double* idd_out, double* proxy_out) {
    const double* F = m.st[0][0].data();
    const double* f = m.st[0][1].data();
    const double* F1 = m.st[1][0].data();
    const double* f1 = m.st[1][1].data();
    const bool trap = m.p.flags & BFPN_FLAG_TRAPEZOIDAL_YZ;
    const bool cat = m.p.flags & BFPN_FLAG_DOSE_CATASTROPHIC_LOSS;
    double total = 0.0, proxy = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : total, proxy)
    for (int ek = 0; ek < m.Ng; ++ek) {
        double S_mid = 0.5 * (m.S_s[ek] + m.S_s[ek + 1]);
        double slope_w = (m.S_s[ek + 1] - m.S_s[ek]) / 6.0;
        double sigma = std::max(m.sigma[ek], 0.0);
        double E_mid = 0.5 * (m.en[ek] + m.en[ek + 1]);
        double part = 0.0, pp = 0.0;
        for (int s = 0; s < m.nyz; ++s) {
            int iy = s % (m.Ny + 1), iz = s / (m.Ny + 1);
            double w = 1.0;
            if (trap) {
                if (iy == 0 || iy == m.Ny) w *= 0.5;
                if (iz == 0 || iz == m.Nz) w *= 0.5;
            }
            for (int a = 0; a < m.NA; ++a) {
                size_t id = m.idx(ek, s, a);
                double psi1 = F[id] + F1[id];
                double psi2 = f[id] + f1[id];
                double dose = psi1 * S_mid * m.dg + psi2 * slope_w * m.dg;
                if (cat) dose += psi1 * E_mid * sigma * m.dg + psi2 * (m.en[ek + 1] - m.en[ek]) * sigma * m.dg / 6.0;
                part += w * dose / m.p.density;
                pp += f[id];
            }
        }
        total += part;
        proxy += pp;
    }
    *idd_out = total * m.du * m.dv * m.dy * m.dz;
    *proxy_out = proxy * m.dg;
}

// energyMomentKernel (bfpm_solver.cu:311-360): per group, integrals of psi^1
// and psi^2 over y, z, u, v.
static void energy_moments(const Model& m, double* out) {
#pragma omp parallel for schedule(static)
    for (int ek = 0; ek < m.Ng; ++ek) {
        double s1 = 0.0, s2 = 0.0;
        for (size_t l = 0; l < m.per_e; ++l) {
            size_t id = ek * m.per_e + l;
            s1 += m.st[0][0][id] + m.st[1][0][id];
            s2 += m.st[0][1][id] + m.st[1][1][id];
        }
        double w = m.du * m.dv * m.dy * m.dz;
        out[2 * ek] = s1 * w;
        out[2 * ek + 1] = s2 * w;
    }
}

// spotDosePlaneKernel (bfpm_solver.cu:433-475): per (y, z) position, the Eq.
// 24 dose of primary + secondary over groups and angles, times du dv.
static void spot_plane(const Model& m, double* plane) {
    const bool cat = m.p.flags & BFPN_FLAG_DOSE_CATASTROPHIC_LOSS;
#pragma omp parallel for schedule(static)
    for (int s = 0; s < m.nyz; ++s) {
        double sum = 0.0;
        for (int ek = 0; ek < m.Ng; ++ek) {
            double S_mid = 0.5 * (m.S_s[ek] + m.S_s[ek + 1]);
            double slope_w = (m.S_s[ek + 1] - m.S_s[ek]) / 6.0;
            for (int a = 0; a < m.NA; ++a) {
                size_t id = m.idx(ek, s, a);
                double psi1 = m.st[0][0][id] + m.st[1][0][id];
                double psi2 = m.st[0][1][id] + m.st[1][1][id];
                double dose = psi1 * S_mid * m.dg + psi2 * slope_w * m.dg;
                if (cat) {
                    double sigma = std::max(m.sigma[ek], 0.0);
                    double E_mid = 0.5 * (m.en[ek] + m.en[ek + 1]);
                    dose += psi1 * E_mid * sigma * m.dg + psi2 * (m.en[ek + 1] - m.en[ek]) * sigma * m.dg / 6.0;
                }
                sum += dose / m.p.density;
            }
        }
        plane[s] = sum * m.du * m.dv;
    }
}

// litePrimaryEnergyStepKernel, bfpm_solver.cu:593-620 (stepLitePrimary,
// 3396-3416): psi^1 only, first-order upwind in energy with attenuation.
static void lite_step(Model& m) {
    double* F = m.st[0][0].data();
#pragma omp parallel for schedule(static)
    for (long long lane = 0; lane < static_cast<long long>(m.per_e); ++lane) {
        double next_F = 0.0;
        for (int ek = m.Ng - 1; ek >= 0; --ek) {
            size_t id = static_cast<size_t>(ek) * m.per_e + lane;
            double Fg = std::max(F[id], 0.0);
            double sig = std::max(m.sigma[ek], 0.0);
            double S_lo = std::max(m.S_s[ek], 0.0);
            double S_hi = std::max(m.S_s[ek + 1], 0.0);
            double denom = 1.0 / m.dt + S_lo / m.dg + sig;
            double F_val = (Fg / m.dt + S_hi / m.dg * next_F) / std::max(denom, EPSILON);
            F[id] = std::max(F_val, 0.0);
            next_F = F[id];
        }
    }
}

// integratedDepthDoseLiteKernel, bfpm_solver.cu:523-591
// (computeIntegratedDepthDoseLite, 3528-3558): psi^1 only.
static double lite_idd(const Model& m) {
    const double* F = m.st[0][0].data();
    const bool trap = m.p.flags & BFPN_FLAG_TRAPEZOIDAL_YZ;
    const bool cat = m.p.flags & BFPN_FLAG_DOSE_CATASTROPHIC_LOSS;
    double total = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : total)
    for (int ek = 0; ek < m.Ng; ++ek) {
        double S_mid = 0.5 * (m.S_s[ek] + m.S_s[ek + 1]);
        double E_mid = 0.5 * (m.en[ek] + m.en[ek + 1]);
        double part = 0.0;
        for (int s = 0; s < m.nyz; ++s) {
            int iy = s % (m.Ny + 1), iz = s / (m.Ny + 1);
            double w = 1.0;
            if (trap) {
                if (iy == 0 || iy == m.Ny) w *= 0.5;
                if (iz == 0 || iz == m.Nz) w *= 0.5;
            }
            for (int a = 0; a < m.NA; ++a) {
                double Fv = F[m.idx(ek, s, a)];
                double dose = Fv * S_mid * m.dg;
                if (cat) dose += Fv * E_mid * std::max(m.sigma[ek], 0.0) * m.dg;
                part += w * dose / m.p.density;
            }
        }
        total += part;
    }
    return total * m.du * m.dv * m.dy * m.dz;
}

// stepPrimary (bfpm_solver.cu:3238-3311), stepPrimaryEnergyOnly
// (3313-3333), stepSecondary (3335-3394), and the loop body of solve
// (2190-2254).
static void step(Model& m, double* idd_out, double* proxy_out) {
    if (m.p.flags & BFPN_FLAG_LITE_MEMORY) {  // the lite branch of solve, bfpm_solver.cu:2191-2210
        lite_step(m);
        *idd_out = lite_idd(m);
        *proxy_out = 0.0;
        m.steps_done++;
        return;
    }
    const double h = 0.5 * m.dt;
    const unsigned fl = m.p.flags;
    const bool no_tr = fl & BFPN_FLAG_NO_TRANSPORT, no_an = fl & BFPN_FLAG_NO_ANGLE;
    const bool no_clip = fl & BFPN_FLAG_NO_SPATIAL_CLIPPING;
    if (fl & BFPN_FLAG_ENERGY_ONLY) {
        energy_sweep(m, 0, h, nullptr);
        energy_sweep(m, 0, h, nullptr);
    } else {
        energy_sweep(m, 0, h, nullptr);
        if (!no_tr) { transport(m, 0, 0, h, no_clip); transport(m, 0, 1, h, true); }
        if (!no_an) { angle(m, 0, 0, m.dt); angle(m, 0, 1, m.dt); }
        if (!no_tr) { transport(m, 0, 0, h, no_clip); transport(m, 0, 1, h, true); }
        energy_sweep(m, 0, h, nullptr);
    }
    if (!(fl & BFPN_FLAG_ENERGY_ONLY) && !(fl & BFPN_FLAG_PRIMARY_ONLY) && m.steps_done > 0) {
        // The source depends only on the primary, which stepSecondary does not
        // modify: both of its evaluations are identical, so it is built once.
        secondary_source(m);
        energy_sweep(m, 1, h, m.source.data());
        transport(m, 1, 0, h, false);
        transport(m, 1, 1, h, true);
        angle(m, 1, 0, m.dt);
        angle(m, 1, 1, m.dt);
        transport(m, 1, 0, h, false);
        transport(m, 1, 1, h, true);
        energy_sweep(m, 1, h, m.source.data());
    }
    idd(m, idd_out, proxy_out);
    m.steps_done++;
}

}  // namespace orc

using orc::Model;

extern "C" {

void* oracle_create(const bfpn_grid* g, const bfpn_phys* p, const double* mu, int mu_rows,
                    const double* sigma, int sigma_rows, char* err, int err_len) {
    auto* m = new Model();
    m->g = *g;
    m->p = *p;
    m->Ng = g->Ng; m->Ny = g->Ny; m->Nz = g->Nz; m->Nmu = g->Nmu; m->Nom = g->Nom;
    m->nyz = (g->Ny + 1) * (g->Nz + 1);
    m->NA = g->Nmu * g->Nom;
    m->per_e = static_cast<size_t>(m->nyz) * m->NA;
    m->cells = m->per_e * g->Ng;
    orc::compute_deltas(*m);
    if (!orc::build_tables(*m, mu, mu_rows, sigma, sigma_rows) || !orc::init_beam(*m)) {
        if (err && err_len > 0) std::snprintf(err, err_len, "%s", m->err.c_str());
        delete m;
        return nullptr;
    }
    return m;
}

void oracle_destroy(void* h) { delete static_cast<Model*>(h); }

void oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void oracle_use_direct_source(void* h, int on) { static_cast<Model*>(h)->direct_source = on != 0; }

void oracle_step(void* h, int nsteps, double* idd, double* proxy) {
    auto* m = static_cast<Model*>(h);
    for (int i = 0; i < nsteps; ++i) {
        double a = 0, b = 0;
        orc::step(*m, &a, &b);
        if (idd) idd[i] = a;
        if (proxy) proxy[i] = b;
    }
}

int oracle_steps_done(void* h) { return static_cast<Model*>(h)->steps_done; }
unsigned long long oracle_cells(void* h) { return static_cast<Model*>(h)->cells; }

void oracle_get_state(void* h, int species, int coef, double* out) {
    auto* m = static_cast<Model*>(h);
    if (m->st[species][coef].size() != m->cells) {  // lite-memory mode holds psi^1 of the primary only
        std::memset(out, 0, m->cells * sizeof(double));
        return;
    }
    std::memcpy(out, m->st[species][coef].data(), m->cells * sizeof(double));
}

void oracle_set_state(void* h, int species, int coef, const double* in) {
    auto* m = static_cast<Model*>(h);
    if (m->st[species][coef].size() != m->cells) return;
    std::memcpy(m->st[species][coef].data(), in, m->cells * sizeof(double));
}

void oracle_set_steps_done(void* h, int n) { static_cast<Model*>(h)->steps_done = n; }

void oracle_energy(void* h, int species, double dt, int with_source) {
    auto* m = static_cast<Model*>(h);
    orc::energy_sweep(*m, species, dt, with_source ? m->source.data() : nullptr);
}

void oracle_transport(void* h, int species, int coef, double dt, int preserve_sign) {
    orc::transport(*static_cast<Model*>(h), species, coef, dt, preserve_sign != 0);
}

void oracle_angle(void* h, int species, int coef, double dt) {
    orc::angle(*static_cast<Model*>(h), species, coef, dt);
}

void oracle_source(void* h, double* out) {
    auto* m = static_cast<Model*>(h);
    orc::secondary_source(*m);
    if (out) std::memcpy(out, m->source.data(), m->cells * sizeof(double));
}

void oracle_idd(void* h, double* idd, double* proxy) {
    auto* m = static_cast<Model*>(h);
    if (m->p.flags & BFPN_FLAG_LITE_MEMORY) {
        *idd = orc::lite_idd(*m);
        *proxy = 0.0;
        return;
    }
    orc::idd(*m, idd, proxy);
}

void oracle_energy_moments(void* h, double* out) { orc::energy_moments(*static_cast<Model*>(h), out); }

void oracle_spot_plane(void* h, double* out) { orc::spot_plane(*static_cast<Model*>(h), out); }

// Table access by the same ids as bfpn_table_download.  Returns the count
// written, or -1 for an unknown id / too small a buffer.
long long oracle_table(void* h, int which, double* out, unsigned long long n) {
    auto* m = static_cast<Model*>(h);
    std::vector<double> tmp;
    const std::vector<double>* src = nullptr;
    switch (which) {
        case BFPN_TABLE_S_S: src = &m->S_s; break;
        case BFPN_TABLE_T_C: src = &m->T_c; break;
        case BFPN_TABLE_SIG_TRG: src = &m->sig_trg; break;
        case BFPN_TABLE_SIGMA_C: src = &m->sigma; break;
        case BFPN_TABLE_EN: src = &m->en; break;
        case BFPN_TABLE_OMEND: src = &m->Omend; break;
        case BFPN_TABLE_KER_E1: src = &m->ker_e1; break;
        case BFPN_TABLE_KER_E2: src = &m->ker_e2; break;
        case BFPN_TABLE_KER_V: src = &m->ker_v; break;
        case BFPN_TABLE_BAND:
            tmp.resize(2 * static_cast<size_t>(m->Ng));
            for (int i = 0; i < m->Ng; ++i) { tmp[2 * i] = m->beg[i]; tmp[2 * i + 1] = m->end[i]; }
            src = &tmp;
            break;
        case BFPN_TABLE_BEAM_YZA: src = &m->beam_yza; break;
        case BFPN_TABLE_BEAM_E: src = &m->beam_e; break;
        default: return -1;
    }
    if (src->size() > n) return -1;
    std::memcpy(out, src->data(), src->size() * sizeof(double));
    return static_cast<long long>(src->size());
}

// BFPnSolver::initialize file part (bfpm_solver.cu:1435-1480): the first Ng
// rows of data_cross.txt (falling back to data_b.txt / data_a.txt for a
// bone / air directory) and cross_total.txt, read by whitespace-separated
// number extraction.  Returns 0 on success, 1 if a file cannot be opened.
int oracle_read_tables(const char* data_path, int Ng, double* mu, int* mu_rows,
                       double* sigma, int* sigma_rows) {
    std::string dp(data_path);
    std::string mu_path = dp + "/data_cross.txt";
    std::ifstream mf(mu_path);
    if (!mf) {
        size_t slash = dp.find_last_of("/\\");
        std::string mat = dp.substr(slash == std::string::npos ? 0 : slash + 1);
        if (mat == "bone" || mat == "air") {
            mu_path = dp + "/data_" + mat.substr(0, 1) + ".txt";
            mf.clear();
            mf.open(mu_path);
        }
    }
    if (!mf) return 1;
    for (int i = 0; i < Ng * 3; ++i) mu[i] = 0.0;
    int r = 0;
    while (r < Ng && (mf >> mu[r * 3] >> mu[r * 3 + 1] >> mu[r * 3 + 2])) ++r;
    *mu_rows = r;
    std::ifstream sf(dp + "/cross_total.txt");
    if (!sf) return 1;
    int s = 0;
    while (s < Ng && (sf >> sigma[s])) ++s;
    *sigma_rows = s;
    return 0;
}

}  // extern "C"
