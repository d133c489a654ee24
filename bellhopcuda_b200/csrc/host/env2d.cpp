#include "env2d.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "ldi.h"

namespace bhcb {

namespace {

constexpr double kPi = 3.14159265358979323846;
inline double FLT(float f) { return (double)f; }   // reference FL() literal

[[noreturn]] void env_error(const std::string &m) { throw std::runtime_error(m); }

// ------------------------------------------------------------------ reading
// vector read with the -999.9 sub-tabulation markers preset
// (src/common_setup.hpp:370-381 ReadVector)
template<typename T> void read_vector(LdiReader &f, int32_t &n, std::vector<T> &x)
{
    f.record();
    f.read(n);
    if(n <= 0) env_error("vector length must be positive");
    x.assign(std::max(3, n), (T)0);
    x[1] = x[2] = (T)(-999.9f);
    f.record();
    for(int i = 0; i < n; ++i) f.read(x[i]);
}


void read_bdry_file(const std::string &path, BdryIn &b)
{
    LdiReader f(path);
    if(!f.good()) env_error("unable to open boundary file " + path);
    f.record();
    f.read_chars(b.type, 2);
    int32_t n = 0;
    f.record();
    f.read(n);
    if(n < 1) env_error("boundary file " + path + ": bad point count");
    b.r_km.assign(n, 0.0);
    b.z.assign(n, 0.0);
    b.geo.assign(b.type[1] == 'L' ? n : 0, {0, 0, 0, 0, 0});
    for(int i = 0; i < n; ++i) {
        f.record();
        f.read(b.r_km[i]);
        f.read(b.z[i]);
        if(b.type[1] == 'L')
            for(int k = 0; k < 5; ++k) f.read(b.geo[i][k]);
    }
    b.file = true;
}

// 3-D boundary grid (src/module/boundary.hpp:103-148): type, Nx + x (km), Ny +
// y (km), then one record of Nx depths per y
void read_bdry3_file(const std::string &path, Bdry3In &b)
{
    LdiReader f(path);
    if(!f.good()) env_error("unable to open boundary file " + path);
    f.record();
    f.read_chars(b.type, 2);
    int32_t nx = 0, ny = 0;
    read_vector(f, nx, b.x_km);
    subtab(b.x_km, nx);
    b.x_km.resize(nx);
    read_vector(f, ny, b.y_km);
    subtab(b.y_km, ny);
    b.y_km.resize(ny);
    if(nx < 2 || ny < 2) env_error("boundary file " + path + ": need at least 2 x 2 points");
    b.z.assign((size_t)nx * ny, 0.0);
    for(int iy = 0; iy < ny; ++iy) {
        f.record();
        for(int ix = 0; ix < nx; ++ix) f.read(b.z[(size_t)ix * ny + iy]);
    }
    if(b.type[1] == 'L') env_error("3-D bottom provinces ('L') are not supported by this build");
    b.file = true;
}

// hexahedral SSP file (src/module/ssp.hpp:144-186): Nx + x (km), Ny + y (km),
// Nz + z (m), then for each z and y one record of Nx sound speeds
void read_hex_ssp(const std::string &path, EnvInput &in)
{
    LdiReader f(path);
    if(!f.good()) env_error("unable to open hexahedral SSP file " + path);
    int32_t nx = 0, ny = 0, nz = 0;
    f.record(); f.read(nx);
    if(nx < 2) env_error("hexahedral SSP: need at least two points in x, y, z");
    in.hex_x_km.assign(nx, 0.0);
    f.record();
    for(int i = 0; i < nx; ++i) f.read(in.hex_x_km[i]);
    f.record(); f.read(ny);
    if(ny < 2) env_error("hexahedral SSP: need at least two points in x, y, z");
    in.hex_y_km.assign(ny, 0.0);
    f.record();
    for(int i = 0; i < ny; ++i) f.read(in.hex_y_km[i]);
    f.record(); f.read(nz);
    if(nz < 2) env_error("hexahedral SSP: need at least two points in x, y, z");
    in.hex_z.assign(nz, 0.0);
    f.record();
    for(int i = 0; i < nz; ++i) f.read(in.hex_z[i]);
    in.hex_c.assign((size_t)nx * ny * nz, 0.0);
    for(int iz = 0; iz < nz; ++iz)
        for(int iy = 0; iy < ny; ++iy) {
            f.record();
            for(int ix = 0; ix < nx; ++ix) f.read(in.hex_c[((size_t)ix * ny + iy) * nz + iz]);
        }
}

// quad SSP file (src/module/ssp.hpp:122-141): Nr, the Nr profile ranges (km),
// then one record of Nr sound speeds per depth of the .env profile
void read_quad_ssp(const std::string &path, EnvInput &in)
{
    LdiReader f(path);
    if(!f.good()) env_error("unable to open quad SSP file " + path);
    int32_t nr = 0;
    f.record(); f.read(nr);
    if(nr < 2) env_error("quad SSP: at least two profiles are needed");
    in.quad_r_km.assign(nr, 0.0);
    f.record();
    for(int i = 0; i < nr; ++i) f.read(in.quad_r_km[i]);
    const size_t nz = in.ssp_z.size();
    in.quad_c.assign(nz * nr, 0.0);
    for(size_t iz = 0; iz < nz; ++iz) {
        f.record();
        for(int ir = 0; ir < nr; ++ir) f.read(in.quad_c[iz * nr + ir]);
    }
    for(int i = 1; i < nr; ++i)
        if(!(in.quad_r_km[i] > in.quad_r_km[i - 1])) env_error("quad SSP: profile ranges must be monotone increasing");
}

// reflection coefficient file (src/module/reflcoef.hpp:50-75, 129-145): NPts,
// then NPts (theta, |R|, phase) triples in one list-directed record
void read_refl_file(const std::string &path, bool istop, std::vector<std::array<double, 3>> &tab)
{
    const std::string which = istop ? "top" : "bottom";
    LdiReader f(path);
    if(!f.good()) env_error("unable to open " + which + " reflection coefficient file " + path);
    int32_t n = 0;
    f.record(); f.read(n);
    if(n < 1) env_error(which + " reflection coefficient file: no points");
    tab.assign(n, {0.0, 0.0, 0.0});
    f.record();
    for(int i = 0; i < n; ++i)
        for(int k = 0; k < 3; ++k) f.read(tab[i][k]);
    for(int i = 1; i < n; ++i)
        if(!(tab[i][0] > tab[i - 1][0]))
            env_error(which + " reflection coefficients must be monotonically increasing");
}

// the device form: (theta deg, |R|, phase rad) triples (src/module/reflcoef.hpp:155-165)
std::vector<double> refl_table(const std::vector<std::array<double, 3>> &tab)
{
    const double DegRad = kPi / 180.0;
    std::vector<double> t;
    for(const auto &r : tab) {
        t.push_back(r[0]);
        t.push_back(r[1]);
        t.push_back(r[2] * DegRad);
    }
    return t;
}

// ------------------------------------------------------------- preprocessing
double franc_garr(double f, const double fg[4])
{
    double T = fg[0], S = fg[1], pH = fg[2], zb = fg[3];
    double c = FLT(1412.0) + FLT(3.21) * T + FLT(1.19) * S + FLT(0.0167) * zb;
    double a1 = FLT(8.86) / c * std::pow(FLT(10.0), FLT(0.78) * pH - FLT(5.0));
    double p1 = FLT(1.0);
    double f1 = FLT(2.8) * std::sqrt(S / 35) * std::pow(FLT(1.0), FLT(4.0) - FLT(1245.0) / (T + FLT(273.0)));
    double a2 = FLT(21.44) * S / c * (FLT(1.0) + FLT(0.025) * T);
    double p2 = FLT(1.0) - 1.37e-4 * zb + 6.2e-9 * zb * zb;
    double f2 = FLT(8.17) * std::pow(FLT(10.0), FLT(8.0) - FLT(1990.0) / (T + 273))
        / (FLT(1.0) + FLT(0.0018) * (S - FLT(35.0)));
    double p3 = FLT(1.0) - 3.83e-5 * zb + 4.9e-10 * zb * zb;
    double a3 = (T < FLT(20.0))
        ? 4.937e-4 - 2.59e-5 * T + 9.11e-7 * T * T - 1.5e-8 * T * T * T
        : 3.964e-4 - 1.146e-5 * T + 1.45e-7 * T * T - 6.5e-10 * T * T * T;
    return a1 * p1 * (f1 * f * f) / (f1 * f1 + f * f) + a2 * p2 * (f2 * f * f) / (f2 * f2 + f * f)
        + a3 * p3 * f * f;
}

// attenuation -> complex sound speed (src/module/atten.cpp:99-194)
cpxd crci(const EnvInput &in, double freq, double fT, double z, double c, double alpha, char au0,
          char au1)
{
    double freq0 = freq;
    double omega = FLT(2.0) * kPi * freq;
    double aT = 0.0;
    switch(au0) {
    case 'N': aT = alpha; break;
    case 'M': aT = alpha / 8.6858896; break;
    case 'm':
        aT = alpha / 8.6858896;
        if(freq < fT) aT *= std::pow(freq / freq0, 1.0);
        else aT *= (freq / freq0) * std::pow(fT / freq0, 1.0 - FLT(1.0));
        break;
    case 'F': aT = alpha * freq / 8685.8896; break;
    case 'W': if(std::fabs(c) >= DBL_EPSILON) aT = alpha * freq / (8.6858896 * c); break;
    case 'Q': if(std::fabs(c * alpha) >= DBL_EPSILON) aT = omega / (FLT(2.0) * c * alpha); break;
    case 'L': if(std::fabs(c) >= DBL_EPSILON) aT = alpha * omega / c; break;
    }
    if(au1 == 'T') {
        double f2 = (freq / FLT(1000.0)) * (freq / FLT(1000.0));
        double th = FLT(3.3e-3) + FLT(0.11) * f2 / (FLT(1.0) + f2) + FLT(44.0) * f2 / (FLT(4100.0) + f2)
            + FLT(3e-4) * f2;
        aT += th / FLT(8685.8896);
    } else if(au1 == 'F') {
        aT += franc_garr(freq / FLT(1000.0), in.fg) / FLT(8685.8896);
    } else if(au1 == 'B') {
        for(const auto &b : in.bio) {
            if(z >= b[0] && z <= b[1]) {
                double q = 1.0 - (b[2] * b[2]) / (freq * freq);
                aT += (b[4] / (q * q + 1.0 / (b[3] * b[3]))) / FLT(8685.8896);
            }
        }
    }
    aT *= (c * c) / omega;
    return cpxd(c, aT);
}

// de Boor cubic spline with complex ordinates (src/curves.hpp:76-188)
void cspline(const double *tau, cpxd *c1, cpxd *c2, cpxd *c3, cpxd *c4, int n, int ibcbeg, int ibcend)
{
    cpxd g = 0.0;
    int l = n - 1;
    for(int m = 1; m < n; ++m) {
        c3[m] = cpxd(tau[m] - tau[m - 1], FLT(0.0));
        c4[m] = (c1[m] - c1[m - 1]) / c3[m];
    }
    if(ibcbeg == 0) {
        if(n > 2) {
            c4[0] = c3[2];
            c3[0] = c3[1] + c3[2];
            c2[0] = ((c3[1] + FLT(2.0) * c3[0]) * c4[1] * c3[2] + (c3[1] * c3[1]) * c4[2]) / c3[0];
        } else {
            c4[0] = cpxd(1.0, 0.0);
            c3[0] = cpxd(1.0, 0.0);
            c2[0] = FLT(2.0) * c4[1];
        }
    } else if(ibcbeg == 1) {
        c4[0] = cpxd(1.0, 0.0);
        c3[0] = cpxd(0.0, 0.0);
    } else if(ibcbeg == 2) {
        c4[0] = cpxd(2.0, 0.0);
        c3[0] = cpxd(1.0, 0.0);
        c2[0] = FLT(3.0) * c4[1] - c2[0] * c3[1] * FLT(0.5);
    }
    for(int m = 1; m < l; ++m) {
        g = -c3[m + 1] / c4[m - 1];
        c2[m] = g * c2[m - 1] + FLT(3.0) * (c3[m] * c4[m + 1] + c3[m + 1] * c4[m]);
        c4[m] = g * c3[m - 1] + FLT(2.0) * (c3[m] + c3[m + 1]);
    }
    if(ibcend != 1) {
        if(ibcend == 0) {
            if(n == 2 && ibcbeg == 0) {
                c2[n - 1] = c4[n - 1];
            } else if((n == 3 && ibcbeg == 0) || n == 2) {
                c2[n - 1] = FLT(2.0) * c4[n - 1];
                c4[n - 1] = cpxd(1.0, 0.0);
                g = FLT(1.0) / -c4[n - 2];
            } else {
                g = c3[n - 2] + c3[n - 1];
                c2[n - 1] = ((c3[n - 1] + FLT(2.0) * g) * c4[n - 1] * c3[n - 2]
                             + (c3[n - 1] * c3[n - 1]) * (c1[n - 2] - c1[n - 3]) / c3[n - 2]) / g;
                g = -g / c4[n - 2];
                c4[n - 1] = c3[n - 2];
            }
        } else if(ibcend == 2) {
            c2[n - 1] = FLT(3.0) * c4[n - 1] + c2[n - 1] * c3[n - 1] * FLT(0.5);
            c4[n - 1] = cpxd(2.0, 0.0);
            g = FLT(1.0) / -c4[n - 2];
        }
        if(ibcbeg > 0 || n > 2) {
            c4[n - 1] += g * c3[n - 2];
            c2[n - 1] = (g * c2[n - 2] + c2[n - 1]) / c4[n - 1];
        }
    }
    for(int j = l - 1; j >= 0; --j) c2[j] = (c2[j] - c3[j] * c2[j + 1]) / c4[j];
    for(int i = 1; i < n; ++i) {
        cpxd dtau = c3[i];
        cpxd divdf1 = (c1[i] - c1[i - 1]) / dtau;
        cpxd divdf3 = c2[i - 1] + c2[i] - FLT(2.0) * divdf1;
        c3[i - 1] = FLT(2.0) * (divdf1 - c2[i - 1] - divdf3) / dtau;
        c4[i - 1] = (divdf3 / dtau) * (FLT(6.0) / dtau);
    }
    c3[n - 1] = c3[l - 1] + (tau[n - 1] - tau[l - 1]) * c4[l - 1];
    c4[n - 1] = cpxd(0.0, 0.0);
    for(int i = 0; i < l; ++i) {
        double dt = tau[i + 1] - tau[i];
        c4[n - 1] += dt * (c1[i] + dt * (c2[i] * FLT(0.5) + dt * (c3[i] / FLT(6.0) + dt * c4[i] / FLT(24.0))));
    }
    c4[n - 1] /= tau[n - 1] - tau[0];
}

double fp_interior(double d1, double d2, double fp)
{
    if(d1 * d2 > FLT(0.0)) {
        if(d1 > FLT(0.0)) return std::min(std::max(fp, 0.0), 3.0 * std::min(d1, d2));
        return std::max(std::min(fp, 0.0), 3.0 * std::max(d1, d2));
    }
    return 0.0;
}
double fp_left(double d1, double d2, double fp)
{
    if(d1 * fp <= 0.0) return FLT(0.0);
    if((d1 * d2 <= 0.0) && (std::fabs(fp) > std::fabs(3.0 * d1))) return 3.0 * d1;
    return fp;
}

// monotone PCHIP coefficients (src/curves.hpp:206-372)
void pchip(const double *x, const cpxd *y, int n, cpxd *p1, cpxd *p2, cpxd *p3, cpxd *p4)
{
    if(n == 2) {
        p1[0] = y[0];
        p2[0] = (y[1] - y[0]) / (x[1] - x[0]);
        p3[0] = 0.0;
        p4[0] = 0.0;
        return;
    }
    std::vector<cpxd> w1(n), w2(n), w3(n), w4(n);
    for(int i = 0; i < n; ++i) p1[i] = y[i];
    auto hdel = [&](int ix, double &h1, double &h2, cpxd &d1, cpxd &d2) {
        h1 = x[ix] - x[ix - 1];
        h2 = x[ix + 1] - x[ix];
        d1 = (y[ix] - y[ix - 1]) / h1;
        d2 = (y[ix + 1] - y[ix]) / h2;
    };
    double h1, h2;
    cpxd d1, d2, ft;
    hdel(1, h1, h2, d1, d2);
    ft = ((2.0 * h1 + h2) * d1 - h1 * d2) / (h1 + h2);
    p2[0] = cpxd(fp_left(d1.real(), d2.real(), ft.real()), fp_left(d1.imag(), d2.imag(), ft.imag()));
    hdel(n - 2, h1, h2, d1, d2);
    ft = (-h2 * d1 + (h1 + 2.0 * h2) * d2) / (h1 + h2);
    p2[n - 1] = cpxd(fp_left(d2.real(), d1.real(), ft.real()), fp_left(d2.imag(), d1.imag(), ft.imag()));
    for(int i = 0; i < n; ++i) w1[i] = p1[i];
    w2[0] = p2[0];
    w2[n - 1] = p2[n - 1];
    cspline(x, w1.data(), w2.data(), w3.data(), w4.data(), n, 1, 1);
    for(int ix = 1; ix < n - 1; ++ix) {
        hdel(ix, h1, h2, d1, d2);
        p2[ix] = cpxd(fp_interior(d1.real(), d2.real(), w2[ix].real()),
                      fp_interior(d1.imag(), d2.imag(), w2[ix].imag()));
    }
    for(int ix = 0; ix < n - 1; ++ix) {
        double h = x[ix + 1] - x[ix];
        cpxd f1 = p1[ix], f2 = p1[ix + 1], f1p = p2[ix], f2p = p2[ix + 1];
        p3[ix] = (3.0 * (f2 - f1) - h * (2.0 * f1p + f2p)) / (h * h);
        p4[ix] = (h * (f1p + f2p) - 2.0 * (f2 - f1)) / (h * h * h);
    }
}

HsDev make_hs(const EnvInput &in, double freq, double fT, const HsIn &h)
{
    HsDev d{};
    d.bc = h.bc;
    char au0 = in.top_opt[2], au1 = in.top_opt[3];
    if(h.bc == 'A') {
        cpxd cP = crci(in, freq, fT, h.zTemp, h.alphaR, h.alphaI, au0, au1);
        cpxd cS = crci(in, freq, fT, h.zTemp, h.betaR, h.betaI, au0, au1);
        d.cPr = cP.real(); d.cPi = cP.imag();
        d.cSr = cS.real(); d.cSi = cS.imag();
        d.rho = h.rho;
    } else if(h.bc == 'G') {   // grain size (src/module/boundarycond.hpp:179-224)
        double Mz = h.Mz, vr, a2f, rho;
        if(Mz >= FLT(-1.0) && Mz < FLT(1.0)) {
            vr = FLT(0.002709) * Mz * Mz - FLT(0.056452) * Mz + FLT(1.2778);
            rho = FLT(0.007797) * Mz * Mz - FLT(0.17057) * Mz + FLT(2.3139);
        } else if(Mz >= FLT(1.0) && Mz < FLT(5.3)) {
            vr = FLT(-0.0014881) * Mz * Mz * Mz + FLT(0.0213937) * Mz * Mz - FLT(0.1382798) * Mz + FLT(1.3425);
            rho = FLT(-0.0165406) * Mz * Mz * Mz + FLT(0.2290201) * Mz * Mz - FLT(1.1069031) * Mz + FLT(3.0455);
        } else {
            vr = FLT(-0.0024324) * Mz + FLT(1.0019);
            rho = FLT(-0.0012973) * Mz + FLT(1.1565);
        }
        if(Mz >= FLT(-1.0) && Mz < FLT(0.0)) a2f = FLT(0.4556);
        else if(Mz >= FLT(0.0) && Mz < FLT(2.6)) a2f = FLT(0.4556) + FLT(0.0245) * Mz;
        else if(Mz >= FLT(2.6) && Mz < FLT(4.5)) a2f = FLT(0.1978) + FLT(0.1245) * Mz;
        else if(Mz >= FLT(4.5) && Mz < FLT(6.0)) a2f = FLT(8.0399) - FLT(2.5228) * Mz + FLT(0.20098) * Mz * Mz;
        else if(Mz >= FLT(6.0) && Mz < FLT(9.5)) a2f = FLT(0.9431) - FLT(0.2041) * Mz + FLT(0.0117) * Mz * Mz;
        else a2f = FLT(0.0601);
        double aR = vr * FLT(1500.0);
        double aI = a2f * (vr / FLT(1000.0)) * FLT(1500.0) * std::log(FLT(10.0)) / (FLT(40.0) * kPi);
        cpxd cP = crci(in, freq, fT, h.zTemp, aR, aI, 'L', ' ');
        d.cPr = cP.real(); d.cPi = cP.imag();
        d.rho = rho;
    }
    return d;
}

// src/module/boundary.hpp:180-226 (extension), 600-896 (2-D tangents/normals/curvature)
std::vector<BdryPtDev> build_bdry(const EnvInput &in, double freq, const BdryIn &b, bool istop,
                                  double depth, int32_t &curv, int32_t &islong)
{
    const double big = std::sqrt(DBL_MAX) / 1.0e5;
    std::vector<BdryPtDev> bd;
    char type0 = 'L', type1 = 'S';
    if(!b.file) {
        bd.assign(2, BdryPtDev{});
        bd[0].x[0] = -big; bd[0].x[1] = depth;
        bd[1].x[0] = big;  bd[1].x[1] = depth;
    } else {
        type0 = b.type[0];
        type1 = b.type[1];
        int n = (int)b.r_km.size() + 2;
        bd.assign(n, BdryPtDev{});
        for(int i = 1; i < n - 1; ++i) {
            bd[i].x[0] = b.r_km[i - 1];
            bd[i].x[1] = b.z[i - 1];
            if(type1 == 'L') {
                const auto &g = b.geo[i - 1];
                cpxd cP = crci(in, freq, 0, 1.0e20, g[0], g[3], 'W', ' ');
                cpxd cS = crci(in, freq, 0, 1.0e20, g[1], g[4], 'W', ' ');
                bd[i].cPr = cP.real(); bd[i].cPi = cP.imag();
                bd[i].cSr = cS.real(); bd[i].cSi = cS.imag();
                bd[i].rho = g[2];
            }
        }
        bd[0] = bd[1];
        bd[0].x[0] = -big * 0.001;
        bd[n - 1] = bd[n - 2];
        bd[n - 1].x[0] = big * 0.001;
        for(auto &p : bd) { std::memset(p.t, 0, sizeof(p.t)); }
    }
    for(auto &p : bd) p.x[0] *= 1000.0;   // km -> m
    int n = (int)bd.size();
    for(int i = 1; i < n; ++i)
        if(!(bd[i].x[0] > bd[i - 1].x[0]))
            env_error(std::string(istop ? "altimetry" : "bathymetry") + " ranges are not monotonically increasing");
    double negtop = istop ? -1.0 : 1.0;
    std::vector<double> Dx(n, 0.0);
    for(int i = 0; i < n - 1; ++i) {
        double tx = bd[i + 1].x[0] - bd[i].x[0], tz = bd[i + 1].x[1] - bd[i].x[1];
        Dx[i] = tz / tx;
        double len = std::sqrt(tx * tx + tz * tz);
        bd[i].Len = len;
        bd[i].t[0] = tx / len;
        bd[i].t[1] = tz / len;
        bd[i].n[0] = -negtop * bd[i].t[1];
        bd[i].n[1] = negtop * bd[i].t[0];
    }
    curv = type0 == 'C';
    islong = type1 == 'L';
    if(type0 == 'C') {
        for(int i = 1; i < n - 1; ++i) {
            double sss = FLT(0.5);
            bd[i].Nodet[0] = (FLT(1.0) - sss) * bd[i - 1].t[0] + sss * bd[i].t[0];
            bd[i].Nodet[1] = (FLT(1.0) - sss) * bd[i - 1].t[1] + sss * bd[i].t[1];
        }
        bd[0].Nodet[0] = 1.0; bd[0].Nodet[1] = 0.0;
        bd[n - 1].Nodet[0] = 1.0; bd[n - 1].Nodet[1] = 0.0;
        for(int i = 0; i < n; ++i) {
            bd[i].Noden[0] = -negtop * bd[i].Nodet[1];
            bd[i].Noden[1] = negtop * bd[i].Nodet[0];
        }
        for(int i = 0; i < n - 1; ++i) {
            double Dxx = (Dx[i + 1] - Dx[i]) / (bd[i + 1].x[0] - bd[i].x[0]);
            bd[i].kappa = Dxx * bd[i].t[0] * bd[i].t[0] * bd[i].t[0];
        }
    } else {
        for(auto &p : bd) p.kappa = 0.0;
    }
    if(type0 != 'L' && type0 != 'C') env_error("unknown boundary interpolation type");
    return bd;
}

} // namespace

// ---------------------------------------------------------------- read_env
EnvInput read_env_files(const std::string &root, bool o3d)
{
    EnvInput in;
    LdiReader f(root + ".env");
    if(!f.good()) env_error("unable to open environment file " + root + ".env");
    in.o3d = o3d;
    f.record(); f.read(in.title);                               // Title
    f.record(); f.read(in.freq0);                               // Freq0
    int32_t nmedia = 1;
    f.record(); f.read(nmedia);                                 // NMedia
    if(nmedia != 1) env_error("only NMEDIA = 1 is supported");
    f.record(); f.read_chars(in.top_opt, 6);                    // TopOpt
    if(in.top_opt[3] == 'F') {
        f.record();
        for(int k = 0; k < 4; ++k) f.read(in.fg[k]);
    } else if(in.top_opt[3] == 'B') {
        int32_t nb = 0;
        f.record(); f.read(nb);
        in.bio.assign(nb, {0, 0, 0, 0, 0});
        for(int i = 0; i < nb; ++i) {
            f.record();
            for(int k = 0; k < 5; ++k) f.read(in.bio[i][k]);
        }
    }
    if(in.top_opt[5] == 'B') env_error("broadband option 'B' is not supported by the reference either");
    // values recycled from the top halfspace to the SSP and the bottom halfspace
    // (src/api.cpp:254-260)
    double rec[5] = {FLT(1500.0), FLT(0.0), FLT(1.0), FLT(0.0), FLT(0.0)};
    in.top.bc = in.top_opt[1];
    if(in.top.bc == 'A') {                                      // BoundaryCondTop
        f.record(); f.read(in.top.zTemp);
        for(int k = 0; k < 5; ++k) f.read(rec[k]);
        in.top.alphaR = rec[0]; in.top.betaR = rec[1]; in.top.rho = rec[2];
        in.top.alphaI = rec[3]; in.top.betaI = rec[4];
    } else if(in.top.bc == 'G') {
        f.record(); f.read(in.top.zTemp); f.read(in.top.Mz);
    }
    {                                                           // SSP
        int32_t npts = 0;
        double sigma = 0;
        f.record(); f.read(npts); f.read(sigma); f.read(in.bot_depth);
        char st = in.top_opt[0];
        if(st != 'A') {
            for(int guard = 0;; ++guard) {
                if(guard > 100001) env_error("number of SSP points exceeds limit");
                double z = 0;
                f.record();
                f.read(z);
                for(int k = 0; k < 5; ++k) f.read(rec[k]);
                in.ssp_z.push_back(z);
                in.alphaR.push_back(rec[0]); in.betaR.push_back(rec[1]); in.rho.push_back(rec[2]);
                in.alphaI.push_back(rec[3]); in.betaI.push_back(rec[4]);
                if(std::fabs(z - in.bot_depth) < FLT(100.0) * FLT_EPSILON) break;
            }
        } else {
            in.ssp_z = {0.0, in.bot_depth};
        }
        if(st == 'H') {
            if(!o3d) env_error("hexahedral SSP ('H') needs a 3-D run");
            read_hex_ssp(root + ".ssp", in);
        } else if(st == 'Q') {
            if(o3d) env_error("quad SSP ('Q'): 2-D profile not supported in 3-D or Nx2D mode");
            read_quad_ssp(root + ".ssp", in);
        }
    }
    f.record(); f.read_chars(in.bot_opt, 6);                    // BotOpt
    double bsigma = 0;
    f.read(bsigma);
    in.bot.bc = in.bot_opt[0];
    if(in.bot.bc == 'A') {                                      // BoundaryCondBot
        f.record(); f.read(in.bot.zTemp);
        for(int k = 0; k < 5; ++k) f.read(rec[k]);
        in.bot.alphaR = rec[0]; in.bot.betaR = rec[1]; in.bot.rho = rec[2];
        in.bot.alphaI = rec[3]; in.bot.betaI = rec[4];
    } else if(in.bot.bc == 'G') {
        f.record(); f.read(in.bot.zTemp); f.read(in.bot.Mz);
    }
    if(o3d) {                                                   // SxSy
        read_vector(f, in.nsx, in.sx_km);
        read_vector(f, in.nsy, in.sy_km);
    }
    read_vector(f, in.nsz, in.sz);                              // SzRz
    read_vector(f, in.nrz, in.rz);
    read_vector(f, in.nrr, in.rr_km);                           // RcvrRanges
    if(o3d) read_vector(f, in.ntheta, in.theta_deg);            // RcvrBearings
    f.record(); f.read_chars(in.run_type, 7);                   // RunType
    {                                                           // RayAnglesElevation
        f.record();
        f.read(in.nalpha);
        if(in.top_opt[5] == 'I') f.read(in.isingle);
        int n = in.nalpha;
        in.alpha_deg.assign(std::max(3, std::max(n, 2)), 0.0);
        if(n > 2) in.alpha_deg[2] = FLT(-999.9);
        f.record();
        int nread = n == 0 ? 2 : n;
        for(int i = 0; i < nread; ++i) f.read(in.alpha_deg[i]);
    }
    if(o3d) {                                                   // RayAnglesBearing
        f.record();
        f.read(in.nbeta);
        if(in.top_opt[5] == 'I') f.read(in.isingle_beta);
        int n = in.nbeta;
        if(n < 0) env_error("number of beams in bearing must not be negative");
        in.beta_deg.assign(std::max(3, n), 0.0);
        if(n > 2) in.beta_deg[2] = FLT(-999.9);
        f.record();
        const int nread = n == 0 ? 2 : n;   // 0: the count is chosen in preprocessing
        for(int i = 0; i < nread; ++i) f.read(in.beta_deg[i]);
    }
    f.record();                                                 // BeamInfo
    if(o3d) {
        f.read(in.deltas); f.read(in.box_x_km); f.read(in.box_y_km); f.read(in.box_z);
    } else {
        f.read(in.deltas); f.read(in.box_z); f.read(in.box_r_km);
    }
    if(in.run_type[0] != 'R' && (in.run_type[1] == 'C' || in.run_type[1] == 'R')) {
        if(o3d) env_error("Cerveny beams are not supported in 3-D (the reference rejects them too)");
        f.record();
        f.read_chars(in.cerv_type, 2);
        f.read(in.eps_mult);
        f.read(in.rloop);
        f.record();
        f.read(in.nimage);
        f.read(in.ibeam_window);
        std::string comp;
        if(f.read(comp) && !comp.empty()) in.component = comp[0];
    }
    if(o3d) {
        if(in.top_opt[4] == '~' || in.top_opt[4] == '*') read_bdry3_file(root + ".ati", in.ati3);
        if(in.bot_opt[1] == '~' || in.bot_opt[1] == '*') read_bdry3_file(root + ".bty", in.bty3);
    } else {
        if(in.top_opt[4] == '~' || in.top_opt[4] == '*') read_bdry_file(root + ".ati", in.ati);
        if(in.bot_opt[1] == '~' || in.bot_opt[1] == '*') read_bdry_file(root + ".bty", in.bty);
    }
    if(in.bot.bc == 'F') read_refl_file(root + ".brc", false, in.brc);   // BRC
    if(in.top.bc == 'F') read_refl_file(root + ".trc", true, in.trc);    // TRC
    if(in.run_type[2] == '*') {                                 // SBP
        LdiReader s(root + ".sbp");
        if(!s.good()) env_error("unable to open source beam pattern file");
        int32_t n = 0;
        s.record(); s.read(n);
        in.sbp.assign(n, {0, 0});
        for(int i = 0; i < n; ++i) { s.record(); s.read(in.sbp[i][0]); s.read(in.sbp[i][1]); }
    }
    return in;
}

// 1-D SSP tables (src/module/ssp.hpp:453-545, src/curves.hpp:76-372), shared
// by the 2-D and 3-D preprocessing
struct Ssp1d {
    std::vector<double> z, rho, c, cz, n2, n2z, coef;
};
void build_ssp1d(const EnvInput &in, double freq, double fT, char st, Ssp1d &t)
{
    int n = (int)in.ssp_z.size();
    if(n < 2) env_error("the SSP must have at least 2 points");
    for(int i = 1; i < n; ++i)
        if(!(in.ssp_z[i] > in.ssp_z[i - 1])) env_error("SSP depths must be monotone increasing");
    t.z = in.ssp_z;
    t.rho = in.rho.empty() ? std::vector<double>(n, 1.0) : in.rho;
    t.c.assign(2 * n, 0.0);
    t.cz.assign(2 * n, 0.0);
    t.n2.assign(2 * n, 0.0);
    t.n2z.assign(2 * n, 0.0);
    t.coef.assign(8 * n, 0.0);
    if(st != 'A') {
        std::vector<cpxd> c(n), cz(n, cpxd(NAN, NAN));
        for(int i = 0; i < n; ++i) {
            c[i] = crci(in, freq, fT, in.ssp_z[i], in.alphaR[i], in.alphaI[i], in.top_opt[2], in.top_opt[3]);
            if(i > 0) cz[i - 1] = (c[i] - c[i - 1]) / (in.ssp_z[i] - in.ssp_z[i - 1]);
        }
        for(int i = 0; i < n; ++i) {
            t.c[2 * i] = c[i].real(); t.c[2 * i + 1] = c[i].imag();
            t.cz[2 * i] = cz[i].real(); t.cz[2 * i + 1] = cz[i].imag();
        }
        if(st == 'N') {
            std::vector<cpxd> n2(n);
            for(int i = 0; i < n; ++i) n2[i] = FLT(1.0) / (c[i] * c[i]);
            for(int i = 0; i < n; ++i) { t.n2[2 * i] = n2[i].real(); t.n2[2 * i + 1] = n2[i].imag(); }
            for(int i = 1; i < n; ++i) {
                cpxd d = (n2[i] - n2[i - 1]) / (in.ssp_z[i] - in.ssp_z[i - 1]);
                t.n2z[2 * (i - 1)] = d.real(); t.n2z[2 * (i - 1) + 1] = d.imag();
            }
        } else if(st == 'S' || st == 'P') {
            std::vector<cpxd> k0(n), k1(n), k2(n), k3(n);
            if(st == 'S') {
                for(int i = 0; i < n; ++i) k0[i] = c[i];
                cspline(in.ssp_z.data(), k0.data(), k1.data(), k2.data(), k3.data(), n, 0, 0);
            } else {
                pchip(in.ssp_z.data(), c.data(), n, k0.data(), k1.data(), k2.data(), k3.data());
            }
            const std::vector<cpxd> *K[4] = {&k0, &k1, &k2, &k3};
            for(int k = 0; k < 4; ++k)
                for(int i = 0; i < n; ++i) {
                    t.coef[2 * (k * n + i)] = (*K[k])[i].real();
                    t.coef[2 * (k * n + i) + 1] = (*K[k])[i].imag();
                }
        }
    }
}

// -------------------------------------------------------------- preprocess
EnvTables preprocess(const EnvInput &in, double freq)
{
    EnvTables t;
    t.freq0 = freq;
    std::memcpy(t.run_type, in.run_type, 7);
    // RunType validation / normalisation (src/module/runtype.hpp:53-78)
    switch(t.run_type[0]) {
    case 'C': case 'S': case 'I': case 'A': case 'a': case 'E': case 'V': case 'v': case 'R': break;
    default: env_error("unknown RunType");
    }
    const bool ray_run = t.run_type[0] == 'R';
    switch(t.run_type[1]) {
    case 'C': case 'R': case 'S': case 'b': case 'B': case 'g': break;
    default: t.run_type[1] = 'G';
    }
    if(t.run_type[3] != 'X') t.run_type[3] = 'R';
    if(t.run_type[4] != 'I') t.run_type[4] = 'R';
    if(t.run_type[5] != ' ' && t.run_type[5] != '2') env_error("3-D environment given to the 2-D reader");
    std::memcpy(t.beam_type, "G S ", 4);                       // MoveBeamType (module/beaminfo.hpp:240-244)
    t.beam_type[0] = t.run_type[1];
    t.beam_type[3] = t.run_type[6];
    char bt = t.beam_type[0];
    if(bt == 'C' || bt == 'R') {                                 // Cerveny (module/beaminfo.hpp:79-90,130-139)
        t.beam_type[1] = in.cerv_type[0];
        t.beam_type[2] = in.cerv_type[1];
        if(!ray_run && t.beam_type[2] != 'D' && t.beam_type[2] != 'Z' && t.beam_type[2] != 'S')
            env_error(std::string("unknown curvature condition '") + t.beam_type[2] + "'");
        if(!ray_run && t.run_type[0] != 'C' && t.run_type[0] != 'S' && t.run_type[0] != 'I')
            env_error("Cerveny influence does not support eigenrays or arrivals");
    }
    t.eps_mult = in.eps_mult;
    t.rloop = in.rloop;
    t.nimage = in.nimage;
    t.ibeam_window = in.ibeam_window;
    t.component = in.component;
    if(!ray_run && (bt == 'C' || bt == 'R') && (in.nimage < 1 || in.nimage > 3))
        env_error("Cerveny beams: the number of images must be 1, 2 or 3");

    char st = in.top_opt[0];
    switch(st) {
    case 'N': t.ssp_type = SSP_N2LINEAR; break;
    case 'C': t.ssp_type = SSP_CLINEAR; break;
    case 'S': t.ssp_type = SSP_CUBIC; break;
    case 'P': t.ssp_type = SSP_PCHIP; break;
    case 'A': t.ssp_type = SSP_ANALYTIC; break;
    case 'Q': t.ssp_type = SSP_QUAD; break;
    default: env_error("unknown SSP type");
    }
    if(in.top.bc != 'V' && in.top.bc != 'R' && in.top.bc != 'A' && in.top.bc != 'G' && in.top.bc != 'F')
        env_error("top boundary condition not supported by this build");
    if(in.bot.bc != 'V' && in.bot.bc != 'R' && in.bot.bc != 'A' && in.bot.bc != 'G' && in.bot.bc != 'F')
        env_error("bottom boundary condition not supported by this build");
    t.brc = refl_table(in.brc);
    t.trc = refl_table(in.trc);
    // fT: 1000 once an 'A' bottom halfspace has been read (module/boundarycond.hpp:37-58)
    double fT = in.bot.bc == 'A' ? FLT(1000.0) : 1.0e20;
    Ssp1d sp;
    build_ssp1d(in, freq, fT, st, sp);
    t.z = sp.z; t.rho = sp.rho; t.c = sp.c; t.cz = sp.cz; t.n2 = sp.n2; t.n2z = sp.n2z; t.coef = sp.coef;
    const int n = (int)in.ssp_z.size();
    if(st == 'Q') {
        // ranges to m and the depth gradient of every profile (src/module/ssp.hpp:456-462,537-545)
        const int nr = (int)in.quad_r_km.size();
        if(nr < 2 || in.quad_c.size() != (size_t)n * nr) env_error("quad SSP: the .ssp file was not read");
        for(double v : in.quad_r_km) t.qr.push_back(v * FLT(1000.0));
        t.qc = in.quad_c;
        t.qcz.assign((size_t)n * nr, 0.0);
        for(int ir = 0; ir < nr; ++ir)
            for(int iz = 1; iz < n; ++iz)
                t.qcz[(size_t)(iz - 1) * nr + ir] = (t.qc[(size_t)iz * nr + ir] - t.qc[(size_t)(iz - 1) * nr + ir])
                    / (in.ssp_z[iz] - in.ssp_z[iz - 1]);
    }
    double top_depth = in.ssp_z[0], bot_depth = in.bot_depth;
    if(std::fabs(in.ssp_z[n - 1] - bot_depth) >= FLT(100.0) * FLT_EPSILON)
        t.warnings.push_back("Ocean bottom must be at last SSP depth");
    t.top = make_hs(in, freq, fT, in.top);
    t.bot = make_hs(in, freq, fT, in.bot);
    t.top_depth = top_depth;
    t.bot_depth = bot_depth;
    t.btop = build_bdry(in, freq, in.ati, true, top_depth, t.top_curv, t.top_long);
    t.bbot = build_bdry(in, freq, in.bty, false, bot_depth, t.bot_curv, t.bot_long);
    for(const auto &p : t.bbot)
        if(p.x[1] > bot_depth) env_error("bathymetry drops below lowest point in the sound speed profile");
    for(const auto &p : t.btop)
        if(p.x[1] < top_depth) env_error("altimetry rises above highest point in the sound speed profile");

    // sources / receivers (module/szrz.hpp:64-125, module/rcvrranges.hpp:74-85)
    t.sz = in.sz;
    subtab(t.sz, in.nsz);
    t.sz.resize(in.nsz);
    std::sort(t.sz.begin(), t.sz.end());
    t.rz = in.rz;
    subtab(t.rz, in.nrz);
    t.rz.resize(in.nrz);
    std::sort(t.rz.begin(), t.rz.end());
    for(auto &v : t.sz) { if(v < top_depth) v = (float)top_depth; if(v > bot_depth) v = (float)bot_depth; }
    for(auto &v : t.rz) { if(v < top_depth) v = (float)top_depth; if(v > bot_depth) v = (float)bot_depth; }
    std::vector<double> rr = in.rr_km;
    subtab(rr, in.nrr);
    rr.resize(in.nrr);
    std::sort(rr.begin(), rr.end());
    for(auto &v : rr) v *= FLT(1000.0);
    for(int i = 1; i < in.nrr; ++i)
        if(!(rr[i] > rr[i - 1])) env_error("receiver ranges are not monotonically increasing");
    t.rr = rr;
    t.delta_r = in.nrr >= 2 ? rr[in.nrr - 1] - rr[in.nrr - 2] : FLT(0.0);
    t.nrz_per_range = t.run_type[4] == 'I' ? 1 : in.nrz;
    if(t.run_type[4] == 'I' && in.nrz != in.nrr)
        t.warnings.push_back("Irregular grid option selected with NRz not equal to Nr");
    if(t.run_type[4] == 'I' && in.nrz < in.nrr)   // receiver ir sits at depth Rz[ir]
        env_error("irregular grid needs at least as many receiver depths as ranges");

    // angles (module/rayangles.hpp:66-190)
    int na = in.nalpha;
    std::vector<double> al = in.alpha_deg;
    if(na == 0) {   // EstimateNumAngles (src/module/rayangles.hpp:212-238)
        double c0 = FLT(1500.0);
        if(ray_run) {
            na = 50;
        } else {
            na = std::max((int)(FLT(0.3) * rr[in.nrr - 1] * freq / c0), 300);
            double dth = std::atan((bot_depth - top_depth) / (FLT(10.0) * rr[in.nrr - 1]));
            na = std::max((int)(kPi / dth), na);
        }
        std::vector<double> a(std::max(3, na), 0.0);
        a[0] = al[0];
        a[1] = al[1];
        if(na > 2) a[2] = FLT(-999.9);
        al = a;
    }
    subtab(al, na);
    al.resize(na);
    std::sort(al.begin(), al.end());
    if(na > 1 && std::fabs(std::fmod(al[na - 1] - al[0], FLT(360.0)))
                     < FLT(10.0) * std::fabs(std::nextafter(360.0, 0.0) - 360.0))
        --na;
    al.resize(na);
    for(int i = 1; i < na; ++i)
        if(!(al[i] > al[i - 1])) env_error("beam angles are not monotonically increasing");
    for(auto &v : al) v *= kPi / 180.0;
    t.alpha = al;
    t.dalpha = na != 1 ? (al[na - 1] - al[0]) / (na - 1) : FLT(0.0);
    t.isingle = in.top_opt[5] == 'I' ? in.isingle : 0;
    if(t.isingle != 0 && (t.isingle < 1 || t.isingle > na)) env_error("selected beam iSingle not in [1, n]");

    // beam box and step (module/beaminfo.hpp:220-237)
    t.box_x = in.box_r_km * FLT(1000.0);
    t.box_y = in.box_z;
    if(t.box_x <= 0.0 || t.box_y <= 0.0) env_error("beam box not set up correctly");
    t.deltas = in.deltas;
    if(std::fabs(t.deltas) < DBL_EPSILON) t.deltas = (bot_depth - top_depth) / FLT(10.0);

    // source beam pattern (module/sbp.hpp:58-67,148-157)
    if(!in.sbp.empty()) {
        for(const auto &p : in.sbp) {
            t.sbp.push_back(p[0]);
            t.sbp.push_back(std::pow(FLT(10.0), p[1] / FLT(20.0)));
        }
    } else {
        t.sbp = {FLT(-180.0), std::pow(FLT(10.0), 0.0 / FLT(20.0)), FLT(180.0), std::pow(FLT(10.0), 0.0 / FLT(20.0))};
    }
    return t;
}

bool EnvTables::same_trajectory_tables(const EnvTables &o) const
{
    // Tables converted from attenuation units by crci differ between
    // frequencies only by rounding when the units are frequency independent
    // (e.g. dB/wavelength); a relative tolerance of 1e-12 accepts exactly
    // those cases and rejects genuinely frequency-dependent attenuation.
    auto close = [](double a, double b) {
        if(a == b) return true;
        if(std::isnan(a) && std::isnan(b)) return true;
        return std::fabs(a - b) <= 1e-12 * std::max(std::fabs(a), std::fabs(b));
    };
    auto vclose = [&](const std::vector<double> &a, const std::vector<double> &b) {
        if(a.size() != b.size()) return false;
        for(size_t i = 0; i < a.size(); ++i)
            if(!close(a[i], b[i])) return false;
        return true;
    };
    auto hclose = [&](const HsDev &a, const HsDev &b) {
        return a.bc == b.bc && close(a.cPr, b.cPr) && close(a.cPi, b.cPi) && close(a.cSr, b.cSr)
            && close(a.cSi, b.cSi) && close(a.rho, b.rho);
    };
    auto bclose = [&](const std::vector<BdryPtDev> &a, const std::vector<BdryPtDev> &b) {
        if(a.size() != b.size()) return false;
        for(size_t i = 0; i < a.size(); ++i) {
            const double *x = reinterpret_cast<const double *>(&a[i]);
            const double *y = reinterpret_cast<const double *>(&b[i]);
            for(size_t k = 0; k < sizeof(BdryPtDev) / sizeof(double); ++k)
                if(!close(x[k], y[k])) return false;
        }
        return true;
    };
    // The 2-D halfspace reflection coefficient depends on omega only through
    // cP, cS (the omega factors cancel, src/reflect.hpp:316-350), and the
    // semi-coherent Lloyd-mirror source amplitude depends on omega
    // (src/trace.hpp:148-152), so 'S' runs never share.
    return vclose(c, o.c) && vclose(cz, o.cz) && vclose(n2, o.n2) && vclose(n2z, o.n2z)
        && vclose(coef, o.coef) && vclose(qc, o.qc) && vclose(qr, o.qr) && hclose(top, o.top) && hclose(bot, o.bot) && bclose(btop, o.btop)
        && bclose(bbot, o.bbot) && alpha == o.alpha && run_type[0] != 'S'
        // the other beam types evaluate their beams at the trace frequency
        && (beam_type[0] == 'G' || beam_type[0] == 'B' || beam_type[0] == '^' || beam_type[0] == ' ');
}


// ------------------------------------------------------------ 3-D preprocess
namespace {

// Node normals of a grid boundary, from one-sided differences at the edges and
// centred ones inside, and for a curvilinear ('C') grid the curvatures of each
// cell: depth curvatures from the change of the unscaled node normal across
// the cell, scaled by its length, and angle curvatures from the change of the
// normal's angle in the x-z plane (src/module/boundary.hpp:643-823); zero for
// flat-triangle grids (src/module/boundary.hpp:866-887). The last row and
// column hold no cell and get NaN, never read.
void curvatures3(std::vector<Bdry3Pt> &bd, int nx, int ny, bool curvilinear)
{
    auto P = [&](int ix, int iy) -> Bdry3Pt & { return bd[(size_t)ix * ny + iy]; };
    std::vector<double> nu((size_t)nx * ny * 3), phi((size_t)nx * ny);
    for(int ix = 0; ix < nx; ++ix)
        for(int iy = 0; iy < ny; ++iy) {
            const int x0 = ix == 0 ? 0 : ix - 1, x1 = ix == nx - 1 ? ix : ix + 1;
            const int y0 = iy == 0 ? 0 : iy - 1, y1 = iy == ny - 1 ? iy : iy + 1;
            const double mx = (P(x1, iy).x[2] - P(x0, iy).x[2]) / (P(x1, iy).x[0] - P(x0, iy).x[0]);
            const double my = (P(ix, y1).x[2] - P(ix, y0).x[2]) / (P(ix, y1).x[1] - P(ix, y0).x[1]);
            const double n[3] = {-mx, -my, 1.0};
            const double l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            double *u = &nu[((size_t)ix * ny + iy) * 3];
            for(int k = 0; k < 3; ++k) {
                u[k] = n[k];
                P(ix, iy).noden[k] = n[k] / l;
            }
            phi[(size_t)ix * ny + iy] = std::atan2(n[2], n[0]);
        }
    for(int ix = 0; ix < nx; ++ix)
        for(int iy = 0; iy < ny; ++iy) {
            Bdry3Pt &q = P(ix, iy);
            if(ix == nx - 1 || iy == ny - 1) {
                q.zxx = q.zxy = q.zyy = q.kxx = q.kxy = q.kyy = NAN;
                continue;
            }
            if(!curvilinear) {
                q.zxx = q.zxy = q.zyy = q.kxx = q.kxy = q.kyy = 0.0;
                continue;
            }
            const double *u00 = &nu[((size_t)ix * ny + iy) * 3];
            const double *u10 = &nu[((size_t)(ix + 1) * ny + iy) * 3];
            const double *u01 = &nu[((size_t)ix * ny + iy + 1) * 3];
            const Bdry3Pt &a = P(ix, iy), &bx = P(ix + 1, iy), &by = P(ix, iy + 1);
            q.zxx = -(u10[0] - u00[0]) / (bx.x[0] - a.x[0]);
            const double lx = std::sqrt((bx.x[0] - a.x[0]) * (bx.x[0] - a.x[0]) + (bx.x[2] - a.x[2]) * (bx.x[2] - a.x[2]));
            q.kxx = (phi[(size_t)(ix + 1) * ny + iy] - phi[(size_t)ix * ny + iy]) / lx;
            q.zxy = -(u01[0] - u00[0]) / (by.x[1] - a.x[1]);
            const double ly = std::sqrt((by.x[1] - a.x[1]) * (by.x[1] - a.x[1]) + (by.x[2] - a.x[2]) * (by.x[2] - a.x[2]));
            q.kxy = (phi[(size_t)ix * ny + iy + 1] - phi[(size_t)ix * ny + iy]) / ly;
            q.zyy = -(u01[1] - u00[1]) / (by.x[1] - a.x[1]);
            q.kyy = (phi[(size_t)ix * ny + iy + 1] - phi[(size_t)ix * ny + iy]) / ly;
            const double ln = std::sqrt(u00[0] * u00[0] + u00[1] * u00[1] + u00[2] * u00[2]);
            q.zxx /= ln;
            q.zxy /= ln;
            q.zyy /= ln;
        }
}

// grid boundary with the two triangle normals of each cell
// (src/module/boundary.hpp:56-78 default, 499-523 units, 600-645 normals)
std::vector<Bdry3Pt> build_bdry3(const Bdry3In &b, bool istop, double depth, int32_t &nx, int32_t &ny)
{
    std::vector<Bdry3Pt> bd;
    const double negtop = istop ? -1.0 : 1.0;
    if(!b.file) {
        const double big = 1.0e25;   // BDRYBIG in 3-D (src/boundary.hpp:26-34)
        nx = ny = 2;
        bd.resize(4);
        const double xs[4][2] = {{-big, -big}, {-big, big}, {big, -big}, {big, big}};
        for(int i = 0; i < 4; ++i) {
            bd[i].x[0] = xs[i][0]; bd[i].x[1] = xs[i][1]; bd[i].x[2] = depth;
            bd[i].n1[0] = bd[i].n1[1] = 0.0; bd[i].n1[2] = negtop;
            bd[i].n2[0] = bd[i].n2[1] = 0.0; bd[i].n2[2] = negtop;
        }
        curvatures3(bd, nx, ny, false);
        return bd;
    }
    nx = (int32_t)b.x_km.size();
    ny = (int32_t)b.y_km.size();
    for(int i = 1; i < nx; ++i)
        if(!(b.x_km[i] > b.x_km[i - 1])) env_error("boundary x-coordinates are not monotonically increasing");
    for(int i = 1; i < ny; ++i)
        if(!(b.y_km[i] > b.y_km[i - 1])) env_error("boundary y-coordinates are not monotonically increasing");
    if(b.type[0] != 'R' && b.type[0] != 'C')
        env_error("3-D boundary type must be 'R' (flat triangles) or 'C' (curvilinear)");
    bd.resize((size_t)nx * ny);
    for(int ix = 0; ix < nx; ++ix)
        for(int iy = 0; iy < ny; ++iy) {
            Bdry3Pt &p = bd[(size_t)ix * ny + iy];
            p.x[0] = b.x_km[ix] * 1000.0;
            p.x[1] = b.y_km[iy] * 1000.0;
            p.x[2] = b.z[(size_t)ix * ny + iy];
            for(int k = 0; k < 3; ++k) p.n1[k] = p.n2[k] = NAN;
        }
    auto sub = [](const double *a, const double *c, double *o) { for(int k = 0; k < 3; ++k) o[k] = a[k] - c[k]; };
    auto cross = [](const double *u, const double *v, double *o) {
        o[0] = u[1] * v[2] - u[2] * v[1];
        o[1] = u[2] * v[0] - u[0] * v[2];
        o[2] = u[0] * v[1] - u[1] * v[0];
    };
    for(int ix = 0; ix < nx - 1; ++ix)
        for(int iy = 0; iy < ny - 1; ++iy) {
            const double *p1 = bd[(size_t)ix * ny + iy].x, *p2 = bd[(size_t)(ix + 1) * ny + iy].x;
            const double *p3 = bd[(size_t)(ix + 1) * ny + iy + 1].x, *p4 = bd[(size_t)ix * ny + iy + 1].x;
            double u[3], v[3], n[3];
            Bdry3Pt &q = bd[(size_t)ix * ny + iy];
            sub(p2, p1, u); sub(p3, p1, v); cross(u, v, n);          // triangle 1
            if(istop) for(int k = 0; k < 3; ++k) n[k] = -n[k];
            double l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            for(int k = 0; k < 3; ++k) q.n1[k] = n[k] / l;
            sub(p3, p1, u); sub(p4, p1, v); cross(u, v, n);          // triangle 2
            if(istop) for(int k = 0; k < 3; ++k) n[k] = -n[k];
            l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            for(int k = 0; k < 3; ++k) q.n2[k] = n[k] / l;
        }
    curvatures3(bd, nx, ny, b.type[0] == 'C');
    return bd;
}

// ReadVector's SubTab + Sort (src/common_setup.hpp:368-381)
template<typename T> std::vector<T> tab_sort(std::vector<T> v, int n)
{
    subtab(v, n);
    v.resize(n);
    std::sort(v.begin(), v.end());
    return v;
}

// CheckFix360Sweep (src/common_setup.hpp:258-270)
template<typename T> void fix360(std::vector<T> &a)
{
    int n = (int)a.size();
    if(n > 1 && std::fabs(std::fmod((double)(a[n - 1] - a[0]), FLT(360.0)))
                    < FLT(10.0) * std::fabs(std::nextafter(360.0, 0.0) - 360.0))
        a.resize(n - 1);
}

} // namespace

Env3Tables preprocess3d(const EnvInput &in, double freq)
{
    if(!in.o3d) env_error("the environment was not read as a 3-D run");
    Env3Tables t;
    t.freq0 = freq;
    std::memcpy(t.run_type, in.run_type, 7);
    switch(t.run_type[0]) {   // src/module/runtype.hpp:53-78
    case 'C': case 'S': case 'I': case 'A': case 'a': case 'E': case 'V': case 'v': case 'R': break;
    default: env_error("unknown RunType");
    }
    const bool ray_run3 = t.run_type[0] == 'R';
    if(t.run_type[5] != '3' && t.run_type[5] != '2')
        env_error("3-D runs need RunType(6) = '3' (3-D rays) or '2' (Nx2D)");
    t.nx2d = t.run_type[5] == '2';
    switch(t.run_type[1]) {
    case 'C': case 'R': case 'S': case 'b': case 'B': case 'g': break;
    default: t.run_type[1] = 'G';
    }
    if(t.run_type[3] != 'X') t.run_type[3] = 'R';
    if(t.run_type[4] != 'I') t.run_type[4] = 'R';
    if(t.run_type[4] == 'I') env_error("irregular receiver grids are 2-D only");
    std::memcpy(t.beam_type, "G S ", 4);
    t.beam_type[0] = t.run_type[1];
    t.beam_type[3] = t.run_type[6];
    char bt = t.beam_type[0];
    // ray runs trace geometric rays whatever the beam type (src/mode/ray.cpp:44-86)
    if(!ray_run3 && !(bt == 'G' || bt == 'B' || bt == '^' || bt == ' ' || bt == 'g' || bt == 'b'))
        env_error(std::string("3-D beam type '") + bt + "' is not supported by this build (geometric 'G', 'B', 'g', 'b')");
    if(t.nx2d) {   // Nx2D: ray, TL, arrival and eigen runs with Cartesian geometric beams
        if(!ray_run3 && !(bt == 'G' || bt == 'B' || bt == '^' || bt == ' '))
            env_error(std::string("Nx2D beam type '") + bt + "' is not supported by this build (Cartesian 'G' / 'B')");
        if(t.beam_type[3] == 'S') env_error("Nx2D beam shift is not supported by this build");
    }
    if(t.run_type[3] == 'X') env_error("line sources are 2-D only");

    char st = in.top_opt[0];
    double fT = in.bot.bc == 'A' ? FLT(1000.0) : 1.0e20;
    if(in.top.bc != 'V' && in.top.bc != 'R' && in.top.bc != 'A' && in.top.bc != 'G' && in.top.bc != 'F')
        env_error("top boundary condition not supported by this build");
    if(in.bot.bc != 'V' && in.bot.bc != 'R' && in.bot.bc != 'A' && in.bot.bc != 'G' && in.bot.bc != 'F')
        env_error("bottom boundary condition not supported by this build");
    t.brc = refl_table(in.brc);
    t.trc = refl_table(in.trc);
    double top_depth = in.ssp_z[0], bot_depth = in.bot_depth;
    if(st == 'H') {
        t.ssp_type = SSP_HEXAHEDRAL;
        const int nx = (int)in.hex_x_km.size(), ny = (int)in.hex_y_km.size(), nz = (int)in.hex_z.size();
        for(int i = 1; i < nx; ++i) if(!(in.hex_x_km[i] > in.hex_x_km[i - 1])) env_error("hexahedral SSP x not monotone");
        for(int i = 1; i < ny; ++i) if(!(in.hex_y_km[i] > in.hex_y_km[i - 1])) env_error("hexahedral SSP y not monotone");
        for(int i = 1; i < nz; ++i) if(!(in.hex_z[i] > in.hex_z[i - 1])) env_error("hexahedral SSP z not monotone");
        for(double v : in.hex_x_km) t.hx.push_back(v * 1000.0);
        for(double v : in.hex_y_km) t.hy.push_back(v * 1000.0);
        t.hz = in.hex_z;
        t.hc = in.hex_c;
        t.hcz.assign((size_t)nx * ny * (nz - 1), 0.0);
        for(int ix = 0; ix < nx; ++ix)
            for(int iy = 0; iy < ny; ++iy)
                for(int iz = 1; iz < nz; ++iz)
                    t.hcz[((size_t)ix * ny + iy) * (nz - 1) + iz - 1]
                        = (t.hc[((size_t)ix * ny + iy) * nz + iz] - t.hc[((size_t)ix * ny + iy) * nz + iz - 1])
                          / (t.hz[iz] - t.hz[iz - 1]);
        // SegZToZ (src/module/ssp.hpp:561-585): depths become the grid depths;
        // the density keeps the .env values, undefined past their count
        t.z = t.hz;
        t.rho.assign(nz, NAN);
        for(int i = 0; i < nz && i < (int)in.ssp_z.size(); ++i) t.rho[i] = in.rho.empty() ? 1.0 : in.rho[i];
    } else {
        switch(st) {
        case 'N': t.ssp_type = SSP_N2LINEAR; break;
        case 'C': t.ssp_type = SSP_CLINEAR; break;
        case 'S': t.ssp_type = SSP_CUBIC; break;
        case 'P': t.ssp_type = SSP_PCHIP; break;
        case 'A': env_error("analytic SSP is not supported in 3-D by this build");
        default: env_error("unknown SSP type");
        }
        Ssp1d sp;
        build_ssp1d(in, freq, fT, st, sp);
        t.z = sp.z; t.rho = sp.rho; t.c = sp.c; t.cz = sp.cz; t.n2 = sp.n2; t.n2z = sp.n2z; t.coef = sp.coef;
    }
    t.top = make_hs(in, freq, fT, in.top);
    t.bot = make_hs(in, freq, fT, in.bot);
    t.btop = build_bdry3(in.ati3, true, top_depth, t.top_nx, t.top_ny);
    t.bbot = build_bdry3(in.bty3, false, bot_depth, t.bot_nx, t.bot_ny);
    t.top_curv = in.ati3.file && in.ati3.type[0] == 'C';
    t.bot_curv = in.bty3.file && in.bty3.type[0] == 'C';

    // sources, receivers, bearings (module/sxsy.hpp, szrz.hpp, rcvrranges.hpp, rcvrbearings.hpp)
    if(in.nsx <= 0 || in.nsy <= 0 || in.nsz <= 0) env_error("number of sources must be positive");
    if(in.nrz <= 0 || in.nrr <= 0 || in.ntheta <= 0) env_error("number of receivers / bearings must be positive");

    for(double v : tab_sort(in.sx_km, in.nsx)) t.sx.push_back(v * 1000.0);
    for(double v : tab_sort(in.sy_km, in.nsy)) t.sy.push_back(v * 1000.0);
    t.sz = tab_sort(in.sz, in.nsz);
    t.rz = tab_sort(in.rz, in.nrz);
    for(auto &v : t.sz) { if(v < top_depth) v = (float)top_depth; if(v > bot_depth) v = (float)bot_depth; }
    for(auto &v : t.rz) { if(v < top_depth) v = (float)top_depth; if(v > bot_depth) v = (float)bot_depth; }
    for(double v : tab_sort(in.rr_km, in.nrr)) t.rr.push_back(v * 1000.0);
    for(size_t i = 1; i < t.rr.size(); ++i)
        if(!(t.rr[i] > t.rr[i - 1])) env_error("receiver ranges are not monotonically increasing");
    t.theta = tab_sort(in.theta_deg, in.ntheta);
    fix360(t.theta);

    // angles (module/rayangles.hpp): elevation and bearing fans; a count of 0
    // is chosen as EstimateNumAngles does (src/module/rayangles.hpp:212-238):
    // 50 for ray runs, else from the phase of adjacent beams at the last range
    // (and, in elevation, beams thin against the water depth)
    auto estimate = [&](std::vector<double> v, int n, bool bearing) {
        if(n > 0) return tab_sort(v, n);
        const double rmax = t.rr.back();
        if(ray_run3) {
            n = 50;
        } else {
            n = std::max((int)((bearing ? FLT(0.1) : FLT(0.3)) * rmax * freq / FLT(1500.0)), 300);
            if(!bearing) {
                const double dth = std::atan((bot_depth - top_depth) / (FLT(10.0) * rmax));
                n = std::max((int)(kPi / dth), n);
            }
        }
        std::vector<double> a(std::max(3, n), 0.0);
        a[0] = v[0];
        a[1] = v[1];
        if(n > 2) a[2] = FLT(-999.9);
        return tab_sort(a, n);
    };
    std::vector<double> al = estimate(in.alpha_deg, in.nalpha, false);
    fix360(al);
    std::vector<double> be = estimate(in.beta_deg, in.nbeta, true);
    fix360(be);
    if(t.nx2d && !ray_run3) be = t.theta;   // beams on the receiver radials (src/module/rayangles.hpp:163-179)
    for(size_t i = 1; i < al.size(); ++i) if(!(al[i] > al[i - 1])) env_error("elevation angles are not monotonically increasing");
    for(size_t i = 1; i < be.size(); ++i) if(!(be[i] > be[i - 1])) env_error("bearing angles are not monotonically increasing");
    for(auto &v : al) v *= kPi / 180.0;
    for(auto &v : be) v *= kPi / 180.0;
    t.alpha = al;
    t.beta = be;
    t.dalpha = al.size() != 1 ? (al.back() - al.front()) / (double)(al.size() - 1) : FLT(0.0);
    t.dbeta = be.size() != 1 ? (be.back() - be.front()) / (double)(be.size() - 1) : FLT(0.0);
    t.isingle_alpha = in.top_opt[5] == 'I' ? in.isingle : 0;
    t.isingle_beta = in.top_opt[5] == 'I' ? in.isingle_beta : 0;

    // beam box and step (module/beaminfo.hpp:221-237)
    t.box_x = in.box_x_km * FLT(1000.0);
    t.box_y = in.box_y_km * FLT(1000.0);
    t.box_z = in.box_z;
    if(t.box_x <= 0.0 || t.box_y <= 0.0 || t.box_z <= 0.0) env_error("beam box not set up correctly");
    t.deltas = in.deltas;
    if(std::fabs(t.deltas) < DBL_EPSILON) t.deltas = (bot_depth - top_depth) / FLT(10.0);

    if(!in.sbp.empty()) {
        for(const auto &p : in.sbp) {
            t.sbp.push_back(p[0]);
            t.sbp.push_back(std::pow(FLT(10.0), p[1] / FLT(20.0)));
        }
    } else {
        t.sbp = {FLT(-180.0), 1.0, FLT(180.0), 1.0};
    }
    return t;
}

} // namespace bhcb
