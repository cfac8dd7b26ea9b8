// bfp_solver: command line of the reference (src/main.cu:44-356) on the B200
// solver.  Same flags, defaults, quirks and output files.  Extensions:
//   --lg <MeV>            energy-domain width (fixed 259 in the reference)
//   --precision fp64|mixed
//   --device <n>          CUDA ordinal
//   --print-config        print the parsed run as JSON and exit (no GPU use)
#include "solver.hpp"

#include <algorithm>
#include <cmath>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

namespace {

std::vector<double> parseDepthList(const std::string& text) {
    std::vector<double> values;
    std::stringstream ss(text);
    std::string item;
    while (std::getline(ss, item, ','))
        if (!item.empty()) values.push_back(std::stod(item));
    return values;
}

void printGPUInfo() {
    const int n = bfpn_device_count();
    std::cout << "Found " << n << " CUDA device(s)" << std::endl;
    char buf[1024];
    for (int i = 0; i < n; ++i)
        if (bfpn_device_info(i, buf, sizeof buf) > 0) std::cout << "\n" << buf;
    std::cout << std::endl;
}

void printHelp(const char* prog) {
    std::cout << "Usage: " << prog << " [options]\n"
              << "Options:\n"
              << "  <Nx>             Optional x grid points (default: 4000)\n"
              << "  --data <path>    Data file directory (default: ./data)\n"
              << "  --time <value>   Final simulation time (default: 40.0)\n"
              << "  --energy <MeV>   Incoming beam energy E0 (default: 230.0)\n"
              << "  --sigma-e <MeV>  Initial energy Gaussian sigma (default: 1.0)\n"
              << "  --material <name> Material density preset: water, bone, air\n"
              << "  --rho <value>    Override material density in g/cm^3\n"
              << "  --ny <value>     Y grid cells (paper Figure 3 uses 80)\n"
              << "  --nz <value>     Z grid cells (paper Figure 3 uses 80)\n"
              << "  --ly <cm>        Y domain width (default: 1)\n"
              << "  --lz <cm>        Z domain width (default: 1)\n"
              << "  --lu <value>     U angular domain width (default: 1)\n"
              << "  --lv <value>     V angular domain width (default: 1)\n"
              << "  --lg <MeV>       Energy domain width (default: 259)\n"
              << "  --ng <value>     Energy groups (paper Figure 3 uses 500)\n"
              << "  --nmu <value>    Angular u grid points (paper Figure 3 uses 20)\n"
              << "  --nom <value>    Angular v grid points (paper Figure 3 uses 20)\n"
              << "  --precision <fp64|mixed> Device arithmetic (default: fp64)\n"
              << "  --device <n>     CUDA device ordinal (default: 0)\n"
              << "  --lite-memory    Primary-only low-memory mode for large grid development\n"
              << "  --streaming-full Out-of-core mode: the state in pinned host memory, streamed through the GPU in chunks\n"
              << "  --primary-only   Skip secondary proton evolution/source\n"
              << "  --energy-model <eq15|legacy> Energy update model (default: eq15)\n"
              << "  --eq15-straggling Enable Eq.15 straggling/SIPG terms\n"
              << "  --save-energy-moments Save paper Eq.25 energy-moment diagnostics\n"
              << "  --energy-only    Only advance the primary energy subsystem\n"
              << "  --no-transport   Skip the spatial transport subsystem\n"
              << "  --no-angle       Skip the angular diffusion subsystem\n"
              << "  --no-spatial-clipping Disable positivity clipping in spatial transport\n"
              << "  --profile-steps  Print per-kernel device timing summary\n"
              << "  --discrete-angle-delta Use a quadrature-normalized mono-directional beam\n"
              << "  --normalize-initial-mass Normalize the discrete y/z/u/v/E beam mass\n"
              << "  --trapezoidal-yz Use trapezoidal y/z weights in normalization and IDD\n"
              << "  --dose-catastrophic-loss Include the Eq.24 E*sigma_c*psi dose term (default)\n"
              << "  --stopping-power-dose-only Omit the Eq.24 catastrophic-loss dose term\n"
              << "  --no-cross-section-calibration Use fitted sigma_c directly (default)\n"
              << "  --legacy-cross-section-calibration Apply the legacy empirical sigma_c correction\n"
              << "  --sigma-yz <cm>  Initial transverse Gaussian sigma (default: 0.1)\n"
              << "  --lane-chunk <n> Streaming mode: lanes per energy-sweep chunk (default: 262144)\n"
              << "  --energy-chunk <n> Streaming mode: groups per transport/angle chunk (default: 128)\n"
              << "  --stream-dir <path> Accepted (the streamed state is in pinned host memory)\n"
              << "  --idd-stride <n> Streaming mode: write the IDD every n steps (default: 1)\n"
              << "  --spot-depths <x,...> Save YZ dose planes near requested depths\n"
              << "  --spot-prefix <path> Prefix for spot plane files (default: spot)\n"
              << "  --print-config   Print the parsed run as JSON and exit\n"
              << "  --test           Run in test mode\n"
              << "  --help           Show this help\n";
}

}  // namespace

int main(int argc, char** argv) {
    std::string data_path = "./data";
    bool data_path_set = false;
    std::string material_name;
    double tFinal = 40.0;
    bool test_mode = false, print_config = false;
    GridParams grid;
    PhysicsParams phys;
    double sigma_yz = 0.1;
    try {
        for (int i = 1; i < argc; i++) {
            std::string arg = argv[i];
            const bool has = i + 1 < argc;
            if (arg == "--data" && has) {
                data_path = argv[++i];
                data_path_set = true;
            } else if (arg == "--time" && has) {
                tFinal = std::stod(argv[++i]);
            } else if (arg == "--energy" && has) {
                phys.beam_energy = std::stod(argv[++i]);
            } else if (arg == "--sigma-e" && has) {
                phys.sig_E = std::stod(argv[++i]);
            } else if (arg == "--rho" && has) {
                phys.density = std::stod(argv[++i]);
                phys.energy_density = phys.density;
            } else if (arg == "--ny" && has) {
                grid.Ny = std::stoi(argv[++i]);
            } else if (arg == "--nz" && has) {
                grid.Nz = std::stoi(argv[++i]);
            } else if (arg == "--ly" && has) {
                grid.Ly = std::stod(argv[++i]);
            } else if (arg == "--lz" && has) {
                grid.Lz = std::stod(argv[++i]);
            } else if (arg == "--lu" && has) {
                grid.Lu = std::stod(argv[++i]);
            } else if (arg == "--lv" && has) {
                grid.Lv = std::stod(argv[++i]);
            } else if (arg == "--lg" && has) {
                grid.Lg = std::stod(argv[++i]);
            } else if (arg == "--ng" && has) {
                grid.Ng = std::stoi(argv[++i]);
            } else if (arg == "--nmu" && has) {
                grid.Nmu = std::stoi(argv[++i]);
            } else if (arg == "--nom" && has) {
                grid.Nom = std::stoi(argv[++i]);
            } else if (arg == "--material" && has) {
                std::string m = argv[++i];
                material_name = m;
                if (m == "water") {
                    phys.density = 1.0;
                    phys.energy_density = 1.0;
                } else if (m == "bone") {
                    phys.density = 1.757;
                    phys.energy_density = phys.density;
                } else if (m == "air") {
                    phys.density = 0.001205;
                    phys.energy_density = 0.001205;
                } else {
                    std::cerr << "Unknown material: " << m << std::endl;
                    return 1;
                }
            } else if (arg == "--precision" && has) {
                std::string m = argv[++i];
                if (m == "fp64") phys.precision = BFPN_PREC_FP64;
                else if (m == "mixed") phys.precision = BFPN_PREC_MIXED;
                else {
                    std::cerr << "Unknown precision: " << m << std::endl;
                    return 1;
                }
            } else if (arg == "--device" && has) {
                phys.device = std::stoi(argv[++i]);
            } else if (arg == "--test") {
                test_mode = true;
            } else if (arg == "--print-config") {
                print_config = true;
            } else if (arg == "--lite-memory") {
                phys.lite_memory = true;
            } else if (arg == "--streaming-full") {
                phys.streaming_full = true;
            } else if (arg == "--primary-only") {
                phys.primary_only = true;
            } else if (arg == "--energy-model" && has) {
                std::string m = argv[++i];
                if (m == "legacy") phys.legacy_energy = true;
                else if (m == "eq15") phys.legacy_energy = false;
                else {
                    std::cerr << "Unknown energy model: " << m << std::endl;
                    return 1;
                }
            } else if (arg == "--eq15-straggling") {
                phys.eq15_straggling = true;
            } else if (arg == "--save-energy-moments") {
                phys.save_energy_moments = true;
            } else if (arg == "--energy-only") {
                phys.energy_only = true;
            } else if (arg == "--no-transport") {
                phys.no_transport = true;
            } else if (arg == "--no-angle") {
                phys.no_angle = true;
            } else if (arg == "--no-spatial-clipping") {
                phys.no_spatial_clipping = true;
            } else if (arg == "--no-zero-chunk-skip") {
                phys.no_zero_chunk_skip = true;
            } else if (arg == "--no-fused-stream-boundary") {
                phys.no_fused_stream_boundary = true;
            } else if (arg == "--profile-steps") {
                phys.profile_steps = true;
            } else if (arg == "--discrete-angle-delta") {
                phys.discrete_angle_delta = true;
            } else if (arg == "--normalize-initial-mass") {
                phys.normalize_initial_mass = true;
            } else if (arg == "--trapezoidal-yz") {
                phys.trapezoidal_yz = true;
            } else if (arg == "--dose-catastrophic-loss") {
                phys.dose_catastrophic_loss = true;
            } else if (arg == "--stopping-power-dose-only") {
                phys.dose_catastrophic_loss = false;
            } else if (arg == "--no-cross-section-calibration") {
                phys.calibrate_cross_sections = false;
            } else if (arg == "--legacy-cross-section-calibration") {
                phys.calibrate_cross_sections = true;
            } else if (arg == "--sigma-yz" && has) {
                sigma_yz = std::stod(argv[++i]);
            } else if (arg == "--lane-chunk" && has) {
                phys.streaming_lane_chunk = std::stoi(argv[++i]);
            } else if (arg == "--energy-chunk" && has) {
                phys.streaming_energy_chunk = std::stoi(argv[++i]);
            } else if (arg == "--stream-dir" && has) {
                phys.streaming_dir = argv[++i];
            } else if (arg == "--idd-stride" && has) {
                phys.idd_stride = std::max(1, std::stoi(argv[++i]));
            } else if (arg == "--spot-depths" && has) {
                phys.spot_depths = parseDepthList(argv[++i]);
            } else if (arg == "--spot-prefix" && has) {
                phys.spot_prefix = argv[++i];
            } else if (arg == "--help") {
                printHelp(argv[0]);
                return 0;
            } else if (!arg.empty() && arg[0] != '-') {
                grid.Nx = std::stoi(arg);
            }
        }
    } catch (const std::exception& e) {
        std::cerr << "Error: " << e.what() << std::endl;
        return 1;
    }
    if (!data_path_set && !material_name.empty()) data_path = "BFPn_CPU_Solver/" + material_name;  // main.cu:257-259
    if (phys.lite_memory && phys.streaming_full) {
        std::cerr << "--lite-memory and --streaming-full are mutually exclusive" << std::endl;
        return 1;
    }
    phys.a_1 = 1.0 / 2.0 / sigma_yz / sigma_yz;  // main.cu:294-296
    phys.a_2 = 1.0 / 2.0 / 1e-6 / 1e-6;
    phys.C_c = 1.0 / std::sqrt(2.0 * 3.14159265358979323846 * 0.1 * 1e-6);
    phys.material_name = material_name;
    grid.Lx = 40.0;

    if (print_config) {
        const bfpn_phys cp = toCPhys(phys);
        std::cout.precision(17);
        std::cout << "{\"data_path\": \"" << data_path << "\", \"t_final\": " << tFinal << ", \"Nx\": " << grid.Nx
                  << ", \"Ny\": " << grid.Ny << ", \"Nz\": " << grid.Nz << ", \"Ng\": " << grid.Ng
                  << ", \"Nmu\": " << grid.Nmu << ", \"Nom\": " << grid.Nom << ", \"Lx\": " << grid.Lx
                  << ", \"Ly\": " << grid.Ly << ", \"Lz\": " << grid.Lz << ", \"Lu\": " << grid.Lu
                  << ", \"Lv\": " << grid.Lv << ", \"Lg\": " << grid.Lg << ", \"sig_E\": " << cp.sig_E
                  << ", \"a_1\": " << cp.a_1 << ", \"a_2\": " << cp.a_2 << ", \"beam_energy\": " << cp.beam_energy
                  << ", \"density\": " << cp.density << ", \"energy_density\": " << cp.energy_density
                  << ", \"material\": " << cp.material << ", \"flags\": " << cp.flags
                  << ", \"precision\": " << phys.precision << "}" << std::endl;
        return 0;
    }

    printGPUInfo();
    if (test_mode) {
        std::cout << "Running in test mode..." << std::endl;
        return 0;
    }
    std::cout << "Domain widths: Lx=" << grid.Lx << ", Ly=" << grid.Ly << ", Lz=" << grid.Lz << ", Lu=" << grid.Lu
              << ", Lv=" << grid.Lv << std::endl;
    std::cout << "Initial beam sigmas: yz=" << sigma_yz << " cm, E=" << phys.sig_E << " MeV, angular=1e-6"
              << std::endl;
    std::cout << "Initial quadrature: angle=" << (phys.discrete_angle_delta ? "discrete-delta" : "sampled-gaussian")
              << ", mass normalization=" << (phys.normalize_initial_mass ? "on" : "off")
              << ", y/z trapezoidal weights=" << (phys.trapezoidal_yz ? "on" : "off") << std::endl;
    std::cout << "Dose catastrophic-loss term: " << (phys.dose_catastrophic_loss ? "enabled" : "disabled") << std::endl;
    std::cout << "Cross-section calibration: "
              << (phys.calibrate_cross_sections ? "legacy empirical correction" : "disabled") << std::endl;
    std::cout << "Spatial positivity clipping: " << (phys.no_spatial_clipping ? "disabled" : "enabled") << std::endl;
    try {
        BFPnSolver solver(grid, phys);
        solver.initialize(data_path);
        solver.solve(tFinal);
    } catch (const std::exception& e) {
        std::cerr << "Error: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
