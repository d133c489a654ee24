// In-memory 2-D environments of the C ABI (bhcb_env_desc, the values a
// bhcParams<false> holds after bhc::setup / extsetup_*) converted to and from
// the reader's EnvInput, and the sound speed at a point (bhc::get_ssp,
// include/bhc/bhc.hpp:440-452) from the preprocessed tables.
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/bhcb.h"
#include "env2d.h"

namespace bhcb {

namespace {

template<typename T> std::vector<T> span(const T *p, size_t n)
{
    if(n && !p) throw std::invalid_argument("environment descriptor: an array of nonzero length is NULL");
    return n ? std::vector<T>(p, p + n) : std::vector<T>();
}

void boundary_from(BdryIn &b, const char type[2], int32_t n, const double *r, const double *z, const double *geo)
{
    b.file = n > 0;
    b.type[0] = type[0] ? type[0] : 'L';
    b.type[1] = type[1] ? type[1] : 'S';
    if(!b.file) return;
    if(n < 2) throw std::invalid_argument("environment descriptor: a boundary needs at least 2 points");
    b.r_km = span(r, n);
    b.z = span(z, n);
    b.geo.clear();
    if(b.type[1] == 'L') {
        if(!geo) throw std::invalid_argument("environment descriptor: long-format boundary without geoacoustics");
        for(int32_t i = 0; i < n; ++i) b.geo.push_back({geo[5 * i], geo[5 * i + 1], geo[5 * i + 2], geo[5 * i + 3],
                                                          geo[5 * i + 4]});
    }
}

void halfspace_from(HsIn &h, char bc, const double v[7])
{
    h.bc = bc;
    h.zTemp = v[0];
    h.alphaR = v[1];
    h.betaR = v[2];
    h.rho = v[3];
    h.alphaI = v[4];
    h.betaI = v[5];
    h.Mz = v[6];
}

// the descriptor with the arrays it points into (the descriptor first, so
// that its address is the owner's)
struct OwnedDesc {
    bhcb_env_desc d;
    std::string title;
    std::vector<double> bio, ssp_z, alphaR, betaR, rho, alphaI, betaI;
    std::vector<double> ati_r, ati_z, ati_geo, bty_r, bty_z, bty_geo, sbp, rr_km, alpha_deg;
    std::vector<double> quad_r, quad_c, brc, trc;
    std::vector<float> sz, rz;
};

void flatten(const std::vector<std::array<double, 5>> &v, std::vector<double> &out)
{
    out.clear();
    for(const auto &a : v) out.insert(out.end(), a.begin(), a.end());
}

} // namespace

EnvInput env_from_desc(const bhcb_env_desc &d)
{
    EnvInput in;
    in.o3d = false;
    in.title = d.title ? d.title : "";
    in.freq0 = d.freq0;
    std::memcpy(in.top_opt, d.top_opt, 6);
    std::memcpy(in.bot_opt, d.bot_opt, 6);
    for(int k = 0; k < 4; ++k) in.fg[k] = d.fg[k];
    if(d.nbio < 0) throw std::invalid_argument("environment descriptor: nbio < 0");
    for(int32_t i = 0; i < d.nbio; ++i)
        in.bio.push_back({d.bio[5 * i], d.bio[5 * i + 1], d.bio[5 * i + 2], d.bio[5 * i + 3], d.bio[5 * i + 4]});
    halfspace_from(in.top, d.top_opt[1], d.top_hs);
    halfspace_from(in.bot, d.bot_opt[0], d.bot_hs);
    if(d.nssp < 2) throw std::invalid_argument("environment descriptor: the SSP needs at least 2 nodes");
    in.ssp_z = span(d.ssp_z, d.nssp);
    in.alphaR = span(d.ssp_alphaR, d.nssp);
    in.betaR = span(d.ssp_betaR, d.nssp);
    in.rho = span(d.ssp_rho, d.nssp);
    in.alphaI = span(d.ssp_alphaI, d.nssp);
    in.betaI = span(d.ssp_betaI, d.nssp);
    in.bot_depth = d.bot_depth;
    boundary_from(in.ati, d.ati_type, d.nati, d.ati_r_km, d.ati_z, d.ati_geo);
    boundary_from(in.bty, d.bty_type, d.nbty, d.bty_r_km, d.bty_z, d.bty_geo);
    for(int32_t i = 0; i < d.nsbp; ++i) in.sbp.push_back({d.sbp[2 * i], d.sbp[2 * i + 1]});
    if(d.nsz < 1 || d.nrz < 1 || d.nrr < 1 || d.nalpha < 0)
        throw std::invalid_argument("environment descriptor: source / receiver / angle counts");
    in.nsz = d.nsz;
    in.nrz = d.nrz;
    in.nrr = d.nrr;
    in.nalpha = d.nalpha;
    in.isingle = d.isingle;
    in.sz = span(d.sz, d.nsz);
    in.rz = span(d.rz, d.nrz);
    in.rr_km = span(d.rr_km, d.nrr);
    // vectors are complete: pad to the three slots ReadVector always holds
    while(in.sz.size() < 3) in.sz.push_back(in.sz.back());
    while(in.rz.size() < 3) in.rz.push_back(in.rz.back());
    while(in.rr_km.size() < 3) in.rr_km.push_back(in.rr_km.back());
    if(d.nalpha == 0) {   // estimated count over (first, last)
        in.alpha_deg = d.alpha_deg ? std::vector<double>{d.alpha_deg[0], d.alpha_deg[1]}
                                   : std::vector<double>{-20.0, 20.0};
    } else {
        in.alpha_deg = span(d.alpha_deg, d.nalpha);
    }
    while(in.alpha_deg.size() < 3) in.alpha_deg.push_back(in.alpha_deg.back());
    std::memcpy(in.run_type, d.run_type, 7);
    in.cerv_type[0] = d.cerv_type[0] ? d.cerv_type[0] : ' ';
    in.cerv_type[1] = d.cerv_type[1] ? d.cerv_type[1] : 'S';
    in.deltas = d.deltas;
    in.box_z = d.box_z;
    in.box_r_km = d.box_r_km;
    in.eps_mult = d.eps_mult;
    in.rloop = d.rloop;
    in.nimage = d.nimage;
    in.ibeam_window = d.ibeam_window;
    in.component = d.component ? d.component : 'P';
    if(d.nquad_r > 0) {
        in.quad_r_km = span(d.quad_r_km, d.nquad_r);
        in.quad_c = span(d.quad_c, (size_t)d.nquad_r * d.nssp);
    }
    for(int32_t i = 0; i < d.nbrc; ++i) in.brc.push_back({d.brc[3 * i], d.brc[3 * i + 1], d.brc[3 * i + 2]});
    for(int32_t i = 0; i < d.ntrc; ++i) in.trc.push_back({d.trc[3 * i], d.trc[3 * i + 1], d.trc[3 * i + 2]});
    return in;
}

bhcb_env_desc *desc_from_env(const EnvInput &in)
{
    auto o = std::make_unique<OwnedDesc>();
    bhcb_env_desc &d = o->d;
    std::memset(&d, 0, sizeof d);
    o->title = in.title;
    d.title = o->title.c_str();
    d.freq0 = in.freq0;
    std::memcpy(d.top_opt, in.top_opt, 6);
    std::memcpy(d.bot_opt, in.bot_opt, 6);
    for(int k = 0; k < 4; ++k) d.fg[k] = in.fg[k];
    flatten(in.bio, o->bio);
    d.nbio = (int32_t)in.bio.size();
    d.bio = o->bio.data();
    const HsIn *hs[2] = {&in.top, &in.bot};
    double *dst[2] = {d.top_hs, d.bot_hs};
    for(int k = 0; k < 2; ++k) {
        dst[k][0] = hs[k]->zTemp; dst[k][1] = hs[k]->alphaR; dst[k][2] = hs[k]->betaR; dst[k][3] = hs[k]->rho;
        dst[k][4] = hs[k]->alphaI; dst[k][5] = hs[k]->betaI; dst[k][6] = hs[k]->Mz;
    }
    o->ssp_z = in.ssp_z; o->alphaR = in.alphaR; o->betaR = in.betaR; o->rho = in.rho;
    o->alphaI = in.alphaI; o->betaI = in.betaI;
    d.nssp = (int32_t)in.ssp_z.size();
    d.ssp_z = o->ssp_z.data(); d.ssp_alphaR = o->alphaR.data(); d.ssp_betaR = o->betaR.data();
    d.ssp_rho = o->rho.data(); d.ssp_alphaI = o->alphaI.data(); d.ssp_betaI = o->betaI.data();
    d.bot_depth = in.bot_depth;
    std::memcpy(d.ati_type, in.ati.type, 2);
    std::memcpy(d.bty_type, in.bty.type, 2);
    if(in.ati.file) {
        o->ati_r = in.ati.r_km; o->ati_z = in.ati.z; flatten(in.ati.geo, o->ati_geo);
        d.nati = (int32_t)o->ati_r.size();
        d.ati_r_km = o->ati_r.data(); d.ati_z = o->ati_z.data(); d.ati_geo = o->ati_geo.empty() ? nullptr : o->ati_geo.data();
    }
    if(in.bty.file) {
        o->bty_r = in.bty.r_km; o->bty_z = in.bty.z; flatten(in.bty.geo, o->bty_geo);
        d.nbty = (int32_t)o->bty_r.size();
        d.bty_r_km = o->bty_r.data(); d.bty_z = o->bty_z.data(); d.bty_geo = o->bty_geo.empty() ? nullptr : o->bty_geo.data();
    }
    for(const auto &p : in.sbp) { o->sbp.push_back(p[0]); o->sbp.push_back(p[1]); }
    d.nsbp = (int32_t)in.sbp.size();
    d.sbp = o->sbp.data();
    // complete vectors: SubTab as the reader's ReadVector does
    o->sz = in.sz; subtab(o->sz, in.nsz); o->sz.resize(in.nsz);
    o->rz = in.rz; subtab(o->rz, in.nrz); o->rz.resize(in.nrz);
    o->rr_km = in.rr_km; subtab(o->rr_km, in.nrr); o->rr_km.resize(in.nrr);
    d.nsz = in.nsz; d.nrz = in.nrz; d.nrr = in.nrr;
    d.sz = o->sz.data(); d.rz = o->rz.data(); d.rr_km = o->rr_km.data();
    d.nalpha = in.nalpha;
    d.isingle = in.isingle;
    o->alpha_deg = in.alpha_deg;
    if(in.nalpha > 0) { subtab(o->alpha_deg, in.nalpha); o->alpha_deg.resize(in.nalpha); }
    d.alpha_deg = o->alpha_deg.data();
    std::memcpy(d.run_type, in.run_type, 7);
    std::memcpy(d.cerv_type, in.cerv_type, 2);
    d.deltas = in.deltas; d.box_z = in.box_z; d.box_r_km = in.box_r_km;
    d.eps_mult = in.eps_mult; d.rloop = in.rloop; d.nimage = in.nimage; d.ibeam_window = in.ibeam_window;
    d.component = in.component;
    o->quad_r = in.quad_r_km; o->quad_c = in.quad_c;
    d.nquad_r = (int32_t)o->quad_r.size();
    d.quad_r_km = o->quad_r.data(); d.quad_c = o->quad_c.data();
    for(const auto &t : in.brc) o->brc.insert(o->brc.end(), t.begin(), t.end());
    for(const auto &t : in.trc) o->trc.insert(o->trc.end(), t.begin(), t.end());
    d.nbrc = (int32_t)in.brc.size(); d.ntrc = (int32_t)in.trc.size();
    d.brc = o->brc.data(); d.trc = o->trc.data();
    return &o.release()->d;
}

void free_desc(bhcb_env_desc *d)
{
    delete reinterpret_cast<OwnedDesc *>(d);
}

// Sound speed (real part) at range r, depth z from the preprocessed tables,
// with the tracer's interpolation (src/ssp.hpp:53-212).
double ssp_at(const EnvTables &T, double r, double z)
{
    const std::vector<double> &Z = T.z;
    const int n = (int)Z.size();
    if(n < 2) throw std::invalid_argument("SSP has fewer than 2 nodes");
    int iz = 0;
    while(iz < n - 2 && z >= Z[iz + 1]) ++iz;
    const double dz = z - Z[iz];
    switch(T.ssp_type) {
    case SSP_CLINEAR: return T.c[2 * iz] + dz * T.cz[2 * iz];
    case SSP_N2LINEAR: {
        const double w = dz / (Z[iz + 1] - Z[iz]);
        const std::complex<double> n2((1 - w) * T.n2[2 * iz] + w * T.n2[2 * iz + 2],
                                      (1 - w) * T.n2[2 * iz + 1] + w * T.n2[2 * iz + 3]);
        return (1.0 / std::sqrt(n2)).real();
    }
    case SSP_CUBIC: {
        const double *C = T.coef.data();
        return C[2 * iz] + dz * (C[2 * (n + iz)] + dz * (0.5 * C[2 * (2 * n + iz)] +
                                                          (double)(1.0f / 6.0f) * dz * C[2 * (3 * n + iz)]));
    }
    case SSP_PCHIP: {
        const double *C = T.coef.data();
        return C[2 * iz] + (C[2 * (n + iz)] + (C[2 * (2 * n + iz)] + C[2 * (3 * n + iz)] * dz) * dz) * dz;
    }
    case SSP_QUAD: {
        const int nr = (int)T.qr.size();
        int ir = 0;
        while(ir < nr - 2 && r >= T.qr[ir + 1]) ++ir;
        const double c1 = T.qc[iz * nr + ir] + dz * T.qcz[iz * nr + ir];
        const double c2 = T.qc[iz * nr + ir + 1] + dz * T.qcz[iz * nr + ir + 1];
        double s1 = (r - T.qr[ir]) / (T.qr[ir + 1] - T.qr[ir]);
        s1 = std::min(1.0, std::max(0.0, s1));
        return (1 - s1) * c1 + s1 * c2;
    }
    case SSP_ANALYTIC: {
        const double xt = 2.0 * (z - 1300.0) / 1300.0;
        return 1500.0 * (1.0 + 0.00737 * (xt - 1.0 + std::exp(-xt)));
    }
    default: throw std::invalid_argument("SSP type not evaluated by bhcb_ssp_at");
    }
}

// Sound speed at (x, y, z) of a 3-D environment: the hexahedral grid's
// trilinear interpolation (src/ssp.hpp:220-305: c at the cell's four depth
// columns from c + dz * dc/dz, then blended in x and y), or the 1-D profile in
// depth.
double ssp_at3(const Env3Tables &T, double x, double y, double z)
{
    if(T.ssp_type != SSP_HEXAHEDRAL) {
        EnvTables P;
        P.ssp_type = T.ssp_type;
        P.z = T.z; P.c = T.c; P.cz = T.cz; P.n2 = T.n2; P.n2z = T.n2z; P.coef = T.coef;
        return ssp_at(P, 0.0, z);
    }
    const int nx = (int)T.hx.size(), ny = (int)T.hy.size(), nz = (int)T.hz.size();
    if(nx < 2 || ny < 2 || nz < 2) throw std::invalid_argument("hexahedral SSP grid has fewer than 2 nodes per axis");
    if(x < T.hx[0] || x > T.hx[nx - 1] || y < T.hy[0] || y > T.hy[ny - 1])
        throw std::invalid_argument("point outside the hexahedral SSP grid");
    auto seg = [](const std::vector<double> &g, double v) {
        int i = 0;
        while(i < (int)g.size() - 2 && v >= g[i + 1]) ++i;
        return i;
    };
    const int ix = seg(T.hx, x), iy = seg(T.hy, y), iz = seg(T.hz, z);
    auto c_at = [&](int jx, int jy) {
        return T.hc[((size_t)jx * ny + jy) * nz + iz] + (z - T.hz[iz]) * T.hcz[((size_t)jx * ny + jy) * (nz - 1) + iz];
    };
    const double c11 = c_at(ix, iy), c21 = c_at(ix + 1, iy), c12 = c_at(ix, iy + 1), c22 = c_at(ix + 1, iy + 1);
    const double s1 = std::min(1.0, std::max(0.0, (x - T.hx[ix]) / (T.hx[ix + 1] - T.hx[ix])));
    const double s2 = std::min(1.0, std::max(0.0, (y - T.hy[iy]) / (T.hy[iy + 1] - T.hy[iy])));
    const double c1 = c11 + s2 * (c12 - c11), c2 = c21 + s2 * (c22 - c21);
    return c1 + s1 * (c2 - c1);
}

} // namespace bhcb
