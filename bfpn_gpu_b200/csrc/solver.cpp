// Host C++ mirror of the reference's BFPnSolver on the C ABI.
#include "solver.hpp"

#include <chrono>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <stdexcept>

void GridParams::computeDeltas() {  // bfpm_solver.cu:1116-1127
    dt = Lx / Nx;
    dy = Ly / Ny;
    dz = Lz / Nz;
    dg = Lg / Ng;
    du = Lu / (Nom + 1);
    dv = Lv / (Nmu + 1);
}

bfpn_grid toCGrid(const GridParams& g) {
    bfpn_grid c{};
    c.Nx = g.Nx;
    c.Ny = g.Ny;
    c.Nz = g.Nz;
    c.Ng = g.Ng;
    c.Nmu = g.Nmu;
    c.Nom = g.Nom;
    c.Lx = g.Lx;
    c.Ly = g.Ly;
    c.Lz = g.Lz;
    c.Lu = g.Lu;
    c.Lv = g.Lv;
    c.Lg = g.Lg;
    return c;
}

bfpn_phys toCPhys(const PhysicsParams& p) {
    bfpn_phys c{};
    c.sig_E = p.sig_E;
    c.a_1 = p.a_1;
    c.a_2 = p.a_2;
    c.C_c = p.C_c;
    c.beam_energy = p.beam_energy;
    c.density = p.density;
    c.energy_density = p.energy_density;
    c.material = p.material_name == "bone"    ? BFPN_MATERIAL_BONE
                 : p.material_name == "air"   ? BFPN_MATERIAL_AIR
                 : p.material_name == "water" ? BFPN_MATERIAL_WATER
                                              : BFPN_MATERIAL_NONE;
    uint32_t f = 0;
    if (p.primary_only) f |= BFPN_FLAG_PRIMARY_ONLY;
    if (p.legacy_energy) f |= BFPN_FLAG_LEGACY_ENERGY;
    if (p.eq15_straggling) f |= BFPN_FLAG_EQ15_STRAGGLING;
    if (p.save_energy_moments) f |= BFPN_FLAG_SAVE_ENERGY_MOMENTS;
    if (p.energy_only) f |= BFPN_FLAG_ENERGY_ONLY;
    if (p.no_transport) f |= BFPN_FLAG_NO_TRANSPORT;
    if (p.no_angle) f |= BFPN_FLAG_NO_ANGLE;
    if (p.no_spatial_clipping) f |= BFPN_FLAG_NO_SPATIAL_CLIPPING;
    if (p.discrete_angle_delta) f |= BFPN_FLAG_DISCRETE_ANGLE_DELTA;
    if (p.normalize_initial_mass) f |= BFPN_FLAG_NORMALIZE_INITIAL_MASS;
    if (p.trapezoidal_yz) f |= BFPN_FLAG_TRAPEZOIDAL_YZ;
    if (p.dose_catastrophic_loss) f |= BFPN_FLAG_DOSE_CATASTROPHIC_LOSS;
    if (p.calibrate_cross_sections) f |= BFPN_FLAG_CALIBRATE_CROSS_SECTIONS;
    if (p.lite_memory) f |= BFPN_FLAG_LITE_MEMORY;
    if (p.streaming_full) f |= BFPN_FLAG_STREAMING_FULL;
    c.flags = f;
    return c;
}

void BFPnSolver::check(bfpn_status s, const char* what) {
    if (s == BFPN_OK) return;
    std::ostringstream msg;
    msg << what << ": " << bfpn_status_string(s) << ": " << bfpn_last_error(ctx_);
    throw std::runtime_error(msg.str());
}

BFPnSolver::BFPnSolver(const GridParams& g, const PhysicsParams& p) : grid(g), phys(p) {
    grid.computeDeltas();
    if (phys.streaming_full && (phys.save_energy_moments || !phys.spot_depths.empty()))
        throw std::runtime_error(
            "--save-energy-moments and --spot-depths need the device-resident state; run them without --streaming-full");
    const bfpn_grid cg = toCGrid(grid);
    const bfpn_phys cp = toCPhys(phys);
    uint64_t need = 0;
    if (bfpn_footprint_bytes(&cg, &cp, phys.precision, &need) == BFPN_OK) {
        const double one = static_cast<double>(grid.Ny + 1) * (grid.Nz + 1) * grid.Ng * grid.Nmu * grid.Nom *
                           (phys.precision == BFPN_PREC_FP64 ? 8.0 : 4.0) / 1073741824.0;
        std::cout << "Memory estimate:\n  Mode: "
                  << (phys.lite_memory ? "lite-memory primary-only" : phys.streaming_full ? "streaming-full" : "full")
                  << (phys.streaming_full ? " (pinned host state, device chunks, " : " (device resident, ")
                  << (phys.precision == BFPN_PREC_FP64 ? "fp64" : "mixed fp32/fp64") << ")\n"
                  << std::fixed << std::setprecision(2) << "  One phase-space array: " << one << " GiB\n"
                  << "  Estimated device footprint: " << need / 1073741824.0 << " GiB" << std::defaultfloat
                  << std::setprecision(6) << std::endl;
    }
    bfpn_status s = bfpn_create(&cg, &cp, phys.precision, phys.device, &ctx_);
    if (s != BFPN_OK) {
        std::ostringstream msg;
        msg << bfpn_last_error(nullptr);
        throw std::runtime_error(msg.str());
    }
    if (phys.streaming_full) {
        check(bfpn_set_option(ctx_, BFPN_OPT_LANE_CHUNK, phys.streaming_lane_chunk), "lane chunk");
        check(bfpn_set_option(ctx_, BFPN_OPT_ENERGY_CHUNK, phys.streaming_energy_chunk), "energy chunk");
    }
}

BFPnSolver::~BFPnSolver() { bfpn_destroy(ctx_); }

void BFPnSolver::initialize(const std::string& data_path) {
    std::vector<double> mu(static_cast<size_t>(grid.Ng) * 3), sigma(grid.Ng);
    int32_t mu_rows = 0, sigma_rows = 0;
    if (bfpn_read_tables(data_path.c_str(), grid.Ng, mu.data(), &mu_rows, sigma.data(), &sigma_rows) != BFPN_OK)
        throw std::runtime_error(bfpn_last_error(nullptr));
    check(bfpn_load_tables(ctx_, mu.data(), mu_rows, sigma.data(), sigma_rows), "load tables");
    bfpn_setup_info info{};
    check(bfpn_setup_summary(ctx_, &info), "setup summary");
    std::cout << "Loaded scattering data: " << data_path << " (" << info.mu_rows << " explicit rows, "
              << grid.Ng - info.mu_rows << " zero-filled)\n"
              << "Loaded total cross sections: " << data_path << "/cross_total.txt (" << sigma_rows << " rows)"
              << std::endl;
    std::cout << "Beam-energy sigma_c: group=" << info.beam_group << ", E_mid=" << info.beam_group_energy << " MeV"
              << ", fitted=" << info.sigma_fitted << ", used=" << info.sigma_used << std::endl;
    std::cout << "Discrete beam angle center: |omega_y|=" << info.omega_center_y
              << ", |omega_z|=" << info.omega_center_z << std::endl;
    std::cout << "Initial discrete masses: spatial=" << info.spatial_mass << ", angular=" << info.angular_mass
              << ", energy=" << info.energy_mass << ", scale=" << info.initial_scale << std::endl;
    check(bfpn_init_beam(ctx_), "initial beam");
}

void BFPnSolver::solve(double tFinal) {  // bfpm_solver.cu:2166-2267
    const int max_steps = static_cast<int>(std::ceil(tFinal / grid.dt - 1e-12));
    std::cout << "Starting BFPn solver..." << std::endl;
    std::cout << "Grid: " << grid.Nx << "x" << grid.Ny << "x" << grid.Nz << ", Energy: " << grid.Ng
              << ", Angle: " << grid.Nmu << "x" << grid.Nom << std::endl;
    if (phys.lite_memory)  // bfpm_solver.cu:2185-2187
        std::cout << "Mode: lite-memory primary-only (no secondary, no DG slope, no YZ/angular transport)" << std::endl;
    const int n_angle = grid.Nmu * grid.Nom, nyz = (grid.Ny + 1) * (grid.Nz + 1);
    if (phys.streaming_full)  // bfpm_solver.cu:3134-3140
        std::cout << "Mode: streaming-full out-of-core, lane chunk "
                  << std::max(1, std::min(nyz, phys.streaming_lane_chunk / n_angle)) * n_angle << " (requested "
                  << phys.streaming_lane_chunk << "), energy chunk " << std::max(1, phys.streaming_energy_chunk)
                  << ", IDD stride " << std::max(1, phys.idd_stride) << std::endl;
    idd_history_.clear();
    proxy_history_.clear();
    std::vector<double> moments_history;
    std::vector<double> moment_row(2 * static_cast<size_t>(grid.Ng));
    // lite mode writes neither energy moments nor spot planes (its loop body
    // ends after the IDD, bfpm_solver.cu:2191-2210)
    const bool moments = phys.save_energy_moments && !phys.lite_memory;
    const bool per_step = moments || phys.profile_steps;
    if (phys.profile_steps) check(bfpn_set_profiling(ctx_, 1), "profiling");
    const auto t0 = std::chrono::steady_clock::now();
    double t = 0.0;
    int step = 0;
    std::vector<char> spot_saved(phys.spot_depths.size(), 0);
    while (step < max_steps) {
        int chunk = per_step ? 1 : std::min(100 - step % 100, max_steps - step);
        // end a chunk at the first step after which an unsaved spot plane is due
        // (bfpm_solver.cu:2241-2246, depth accumulated the same way)
        if (!phys.spot_depths.empty() && !phys.lite_memory) {
            double tt = t;
            for (int k = 1; k <= chunk; ++k) {
                tt += grid.dt;
                bool due = false;
                for (size_t i = 0; i < phys.spot_depths.size(); ++i)
                    if (!spot_saved[i] && tt + 0.5 * grid.dt >= phys.spot_depths[i]) due = true;
                if (due) {
                    chunk = k;
                    break;
                }
            }
        }
        std::vector<double> idd(chunk), proxy(chunk);
        check(bfpn_step(ctx_, chunk, idd.data(), proxy.data()), "depth step");
        if (moments) {
            check(bfpn_energy_moments(ctx_, moment_row.data()), "energy moments");
            moments_history.insert(moments_history.end(), moment_row.begin(), moment_row.end());
        }
        for (int i = 0; i < chunk; ++i) {
            idd_history_.push_back(idd[i]);
            proxy_history_.push_back(proxy[i]);
            t += grid.dt;
            ++step;
            if (step % 100 == 0)
                std::cout << "Step " << step << ", t = " << t << "/" << tFinal << ", IDD = " << idd[i] << std::endl;
        }
        for (size_t i = 0; i < phys.spot_depths.size() && !phys.lite_memory; ++i)
            if (!spot_saved[i] && t + 0.5 * grid.dt >= phys.spot_depths[i]) {
                saveSpotPlane(phys.spot_depths[i], t);
                spot_saved[i] = 1;
            }
    }
    const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (phys.streaming_full) {
        // the reference's streaming files: a row every idd_stride steps and the
        // last, the scalar proxy written as 0 (bfpm_solver.cu:3144, 3206-3209)
        const int stride = std::max(1, phys.idd_stride);
        std::ofstream fi("idd_output.txt"), fp("dose_output.txt");
        fi << std::setprecision(17) << "# x_cm value\n";
        fp << std::setprecision(17) << "# x_cm value\n";
        for (size_t i = 0; i < idd_history_.size(); ++i)
            if ((i + 1) % stride == 0 || i + 1 == idd_history_.size()) {
                fi << (i + 1) * grid.dt << " " << idd_history_[i] << "\n";
                fp << (i + 1) * grid.dt << " " << 0.0 << "\n";
            }
    } else {
        saveResults(idd_history_, "idd_output.txt");
        saveResults(proxy_history_, "dose_output.txt");
    }
    if (moments) saveEnergyMoments(moments_history, "energy_moments.txt");
    std::cout << "Solver completed. Paper-style IDD saved to idd_output.txt" << std::endl;
    std::cout << "Diagnostic scalar proxy saved to dose_output.txt" << std::endl;
    if (phys.profile_steps && step > 0) {
        const char* names[BFPN_KERNEL_CLASSES] = {"energy", "transport", "angle", "source angular",
                                                  "source energy", "idd"};
        double ms[BFPN_KERNEL_CLASSES] = {};
        int32_t n[BFPN_KERNEL_CLASSES] = {};
        check(bfpn_kernel_profile(ctx_, ms, n, BFPN_KERNEL_CLASSES), "profile");
        double total = 0.0;
        for (double v : ms) total += v;
        std::cout << std::fixed << std::setprecision(6) << "Step timing summary (" << step << " steps):\n"
                  << "  total       " << seconds << " s, per step " << seconds / step << " s\n";
        for (int k = 0; k < BFPN_KERNEL_CLASSES; ++k)
            std::cout << "  " << std::left << std::setw(15) << names[k] << std::right << ms[k] / 1000.0
                      << " s device, per step " << ms[k] / 1000.0 / step << " s, "
                      << (total > 0 ? 100.0 * ms[k] / total : 0.0) << "%, launches " << n[k] << "\n";
        std::cout << std::defaultfloat << std::setprecision(6) << std::flush;
    }
}

void BFPnSolver::saveResults(const std::vector<double>& values, const std::string& filename) {
    std::ofstream out(filename);  // bfpm_solver.cu:3808-3815
    out << std::setprecision(17);
    out << "# x_cm value\n";
    for (size_t i = 0; i < values.size(); i++) out << (i + 1) * grid.dt << " " << values[i] << "\n";
}

void BFPnSolver::saveSpotPlane(double requested_depth, double actual_depth) {  // bfpm_solver.cu:3560-3612
    if (phys.spot_prefix.empty()) return;
    std::vector<double> plane(static_cast<size_t>(grid.Ny + 1) * (grid.Nz + 1));
    check(bfpn_spot_plane(ctx_, plane.data()), "spot plane");
    std::ostringstream name;
    name << phys.spot_prefix << "_req" << std::fixed << std::setprecision(2) << requested_depth << "_x" << std::fixed
         << std::setprecision(2) << actual_depth << ".txt";
    std::ofstream out(name.str());
    out << "# requested_x_cm " << requested_depth << "\n";
    out << "# actual_x_cm " << actual_depth << "\n";
    out << "# y_cm z_cm dose\n";
    const int Ny1 = grid.Ny + 1, Nz1 = grid.Nz + 1;
    for (int j = 0; j < Nz1; ++j) {
        const double z = -0.5 * grid.Lz + j * grid.dz;
        for (int i = 0; i < Ny1; ++i) {
            const double y = -0.5 * grid.Ly + i * grid.dy;
            out << y << " " << z << " " << plane[j * Ny1 + i] << "\n";
        }
        out << "\n";
    }
    std::cout << "Spot dose plane saved to " << name.str() << std::endl;
}

void BFPnSolver::saveEnergyMoments(const std::vector<double>& values, const std::string& filename) {
    std::ofstream out(filename);  // bfpm_solver.cu:3817-3835
    out << "# step x_cm g psi1_integral psi2_integral\n";
    const size_t per_step = static_cast<size_t>(grid.Ng) * 2;
    if (per_step == 0) return;
    const size_t steps = values.size() / per_step;
    for (size_t st = 0; st < steps; ++st) {
        const double x = (st + 1) * grid.dt;
        const size_t base = st * per_step;
        for (int g = 0; g < grid.Ng; ++g)
            out << (st + 1) << " " << x << " " << g << " " << values[base + 2 * g] << " " << values[base + 2 * g + 1]
                << "\n";
    }
}
