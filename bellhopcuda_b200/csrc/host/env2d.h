// 2-D environment: file reading (EnvInput) and preprocessing into the tables
// the kernels consume (EnvTables).
//
// EnvInput holds the values as the reference's modules hold them after Read
// (src/api.cpp:253-277 runs Title, Freq0, NMedia, TopOpt, BoundaryCondTop,
// SSP, BotOpt, BoundaryCondBot, SzRz, RcvrRanges, RunType, RayAngles,
// BeamInfo, Altimetry, Bathymetry, SBP in this order). preprocess() restates
// the modules' Validate/Preprocess steps (src/module/*.hpp) for one frequency.
#pragma once
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <string>
#include <vector>

#include "../bhcb_internal.h"

namespace bhcb {

using cpxd = std::complex<double>;

struct HsIn {
    char bc = 'V';
    double zTemp = 0, alphaR = 0, betaR = 0, rho = 0, alphaI = 0, betaI = 0, Mz = 0;
};

struct BdryIn {
    bool file = false;
    char type[2] = {'L', 'S'};
    std::vector<double> r_km, z;
    std::vector<std::array<double, 5>> geo;   // long format: alphaR betaR rho alphaI betaI
};

// 3-D boundary grid ('R' .ati/.bty, src/module/boundary.hpp:107-148): depths
// z[ix * ny + iy] at x[ix] (km), y[iy] (km)
struct Bdry3In {
    bool file = false;
    char type[2] = {'R', ' '};
    std::vector<double> x_km, y_km, z;
};

struct EnvInput {
    bool o3d = false;                          // read with the 3-D module list
    std::string title;
    double freq0 = 50.0;
    char top_opt[6] = {'C', 'V', 'W', ' ', ' ', ' '};
    char bot_opt[6] = {'R', ' ', ' ', ' ', ' ', ' '};
    double fg[4] = {20.0, 35.0, 8.0, 0.0};     // Francois-Garrison T S pH z_bar
    std::vector<std::array<double, 5>> bio;    // z1 z2 f0 q a0
    HsIn top, bot;
    std::vector<double> ssp_z, alphaR, betaR, rho, alphaI, betaI;
    double bot_depth = 5000.0;
    BdryIn ati, bty;
    std::vector<std::array<double, 2>> sbp;    // angle (deg), level (dB)
    int32_t nsz = 1, nrz = 1, nrr = 1, nalpha = 0, isingle = 0;
    std::vector<float> sz, rz;                 // as read, before SubTab
    std::vector<double> rr_km, alpha_deg;
    char run_type[7] = {'C', 'G', ' ', 'R', 'R', ' ', ' '};
    double deltas = 0, box_z = 0, box_r_km = 0;
    // Cerveny beams (src/module/beaminfo.hpp:79-90): width and curvature
    // options (Beam->Type[1..2]), epsilon multiplier, rLoop, images, window, component
    char cerv_type[2] = {' ', 'S'};
    double eps_mult = 1.0, rloop = 1.0;
    int32_t nimage = 1, ibeam_window = 4;
    char component = 'P';
    // 3-D only (src/module/sxsy.hpp, rcvrbearings.hpp, rayangles.hpp, beaminfo.hpp)
    int32_t nsx = 1, nsy = 1, ntheta = 1, nbeta = 1, isingle_beta = 0;
    std::vector<double> sx_km, sy_km, theta_deg, beta_deg;
    double box_x_km = 0, box_y_km = 0;
    Bdry3In ati3, bty3;
    // hexahedral SSP (.ssp file, src/module/ssp.hpp:144-190): c[(ix * ny + iy) * nz + iz]
    std::vector<double> hex_x_km, hex_y_km, hex_z, hex_c;
    // quad SSP (.ssp file, src/module/ssp.hpp:122-141): profile ranges (km) and
    // c[iz * nr + ir] at the .env profile's depths
    std::vector<double> quad_r_km, quad_c;
    // tabulated reflection coefficients (.brc / .trc, src/module/reflcoef.hpp:50-75):
    // angle of incidence (deg), |R|, phase (deg)
    std::vector<std::array<double, 3>> brc, trc;
};

struct EnvTables {
    double freq0 = 0;
    int32_t ssp_type = SSP_CLINEAR;
    std::vector<double> z, rho, c, cz, n2, n2z, coef;   // complex tables interleaved
    std::vector<double> qr, qc, qcz;                    // quad SSP: ranges (m), c and dc/dz [iz * nr + ir]
    std::vector<double> brc, trc;                       // reflection tables: (theta deg, |R|, phase rad) triples
    HsDev top{}, bot{};
    int32_t top_curv = 0, bot_curv = 0, top_long = 0, bot_long = 0;
    std::vector<BdryPtDev> btop, bbot;
    std::vector<double> rr, alpha, sbp;
    std::vector<float> rz, sz;
    double dalpha = 0, delta_r = 0, deltas = 0, box_x = 0, box_y = 0;
    char run_type[7];
    char beam_type[4];
    int32_t nrz_per_range = 1, isingle = 0;
    double eps_mult = 1.0, rloop = 1.0, top_depth = 0.0, bot_depth = 0.0;
    int32_t nimage = 1, ibeam_window = 4;
    char component = 'P';
    std::vector<std::string> warnings;
    // true when every frequency-dependent table is identical to other's
    bool same_trajectory_tables(const EnvTables &o) const;
};

// 3-D tables (BELLHOP3D field modes)
struct Bdry3Pt {                 // grid node (x, y, z), the normals of its cell's two triangles, and for
    double x[3], n1[3], n2[3];   // curvilinear grids the node normal and the cell's curvatures
    double noden[3];
    double zxx, zxy, zyy, kxx, kxy, kyy;
};
struct Env3Tables {
    double freq0 = 0;
    int32_t ssp_type = SSP_CLINEAR;          // SSP_HEXAHEDRAL or a 1-D type
    std::vector<double> z, rho, c, cz, n2, n2z, coef;   // 1-D tables (complex interleaved), as in 2-D
    std::vector<double> hx, hy, hz, hc, hcz;             // hexahedral grid (m) and c, dc/dz
    std::vector<double> brc, trc;                        // reflection tables as in 2-D
    HsDev top{}, bot{};
    int32_t top_nx = 2, top_ny = 2, bot_nx = 2, bot_ny = 2;
    int32_t top_curv = 0, bot_curv = 0;
    std::vector<Bdry3Pt> btop, bbot;
    std::vector<double> sx, sy, rr, theta, alpha, beta, sbp;   // m, m, m, deg, rad, rad
    std::vector<float> sz, rz;
    double dalpha = 0, dbeta = 0, deltas = 0, box_x = 0, box_y = 0, box_z = 0;
    int32_t isingle_alpha = 0, isingle_beta = 0;
    char run_type[7];
    char beam_type[4];
    bool nx2d = false;                       // RunType(6) '2': N x 2-D rays in the 3-D ocean
    std::vector<std::string> warnings;
};

// SubTab (src/common_setup.hpp:306-334): FMA sub-tabulation of a vector read
// as (first, last, -999.9 marker)
template<typename T> void subtab(std::vector<T> &x, int n)
{
    const T m999 = (T)(sizeof(T) == 4 ? -999.9f : -999.9);
    const T p01 = (T)(sizeof(T) == 4 ? 0.01f : 0.01);
    if(n >= 3 && x.size() >= 3 && std::fabs(x[2] - m999) < p01) {
        if(std::fabs(x[1] - m999) < p01) x[1] = x[0];
        T dx = (x[1] - x[0]) / (T)(n - 1), x0 = x[0];
        if((int)x.size() < n) x.resize(n);
        for(int i = 0; i < n; ++i) x[i] = std::fma((T)i, dx, x0);
    }
}

EnvInput read_env_files(const std::string &fileroot, bool o3d = false);
EnvTables preprocess(const EnvInput &in, double freq);
Env3Tables preprocess3d(const EnvInput &in, double freq);

} // namespace bhcb

struct bhcb_env_desc;
namespace bhcb {
// in-memory 2-D environments of the C ABI (envdesc.cpp)
EnvInput env_from_desc(const bhcb_env_desc &d);
bhcb_env_desc *desc_from_env(const EnvInput &in);   // owns its arrays; free_desc releases it
void free_desc(bhcb_env_desc *d);
double ssp_at(const EnvTables &T, double r, double z);   // sound speed (m/s) at range r, depth z (m)
double ssp_at3(const Env3Tables &T, double x, double y, double z);   // 3-D: at (x, y, z) (m)

} // namespace bhcb
