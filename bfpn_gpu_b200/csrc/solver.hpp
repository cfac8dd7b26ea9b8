// Host C++ mirror of the reference's solver class and parameter structs
// (src/bfpm_solver.cuh:21-62, 97-253): the same three public steps
// (construct, initialize(data_path), solve(tFinal)) and the same output files,
// on top of the C ABI of include/bfpn_capi.h.  Errors are thrown as
// std::runtime_error, as the reference's host code does.
#pragma once

#include "../../include/bfpn_capi.h"

#include <string>
#include <vector>

// GridParams (bfpm_solver.cuh:21-27).
struct GridParams {
    int Nx = 4000, Ny = 10, Nz = 10, Ng = 500, Nmu = 11, Nom = 11;
    double Lx = 40.0, Ly = 1.0, Lz = 1.0, Lu = 1.0, Lv = 1.0, Lg = 259.0;
    double dt = 0, dy = 0, dz = 0, dg = 0, du = 0, dv = 0;
    void computeDeltas();
};

// PhysicsParams (bfpm_solver.cuh:30-62); `precision` selects FP64 (parity)
// or mixed (float state, double energy recursion and IDD).
struct PhysicsParams {
    double sig_E = 1.0;
    double a_1 = 0.0, a_2 = 0.0;
    double C_c = 0.0;
    double beam_energy = 230.0;
    double density = 1.0;
    double energy_density = 1.0;
    std::string material_name;
    bool lite_memory = false;
    bool streaming_full = false;
    bool primary_only = false;
    bool legacy_energy = false;
    bool eq15_straggling = false;
    bool save_energy_moments = false;
    bool energy_only = false;
    bool no_transport = false;
    bool no_angle = false;
    bool no_spatial_clipping = false;
    bool no_zero_chunk_skip = false;
    bool no_fused_stream_boundary = false;
    bool profile_steps = false;
    bool discrete_angle_delta = false;
    bool normalize_initial_mass = false;
    bool trapezoidal_yz = false;
    bool dose_catastrophic_loss = true;
    bool calibrate_cross_sections = false;
    int streaming_lane_chunk = 262144;
    int streaming_energy_chunk = 128;
    std::string streaming_dir = "/tmp";
    std::vector<double> spot_depths;
    std::string spot_prefix = "spot";
    int idd_stride = 1;
    int precision = BFPN_PREC_FP64;
    int device = 0;
};

bfpn_grid toCGrid(const GridParams& g);
bfpn_phys toCPhys(const PhysicsParams& p);

class BFPnSolver {
public:
    BFPnSolver(const GridParams& g, const PhysicsParams& p);
    ~BFPnSolver();
    BFPnSolver(const BFPnSolver&) = delete;
    BFPnSolver& operator=(const BFPnSolver&) = delete;

    void initialize(const std::string& data_path);
    void solve(double tFinal);

    void saveResults(const std::vector<double>& values, const std::string& filename);
    void saveEnergyMoments(const std::vector<double>& values, const std::string& filename);
    void saveSpotPlane(double requested_depth, double actual_depth);

    const std::vector<double>& iddHistory() const { return idd_history_; }
    const std::vector<double>& proxyHistory() const { return proxy_history_; }
    bfpn_ctx* context() { return ctx_; }

private:
    void check(bfpn_status s, const char* what);

    GridParams grid;
    PhysicsParams phys;
    bfpn_ctx* ctx_ = nullptr;
    std::vector<double> idd_history_, proxy_history_;
};
