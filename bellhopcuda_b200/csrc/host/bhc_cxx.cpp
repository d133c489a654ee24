// The bhc:: C++ surface (include/bhcb/bhc.hpp) over the C ABI (include/bhcb.h).
//
// Follows the reference's API semantics (include/bhc/bhc.hpp:58-452,
// src/api.cpp:194-855): setup fills bhcParams from FileRoot's files or from
// the modules' defaults (src/module/*.hpp Default()), the caller may edit the
// parameters or resize them with extsetup_*, run turns the 2-D parameters into
// an in-memory environment (bhcb_add_env_desc) and fills bhcOutputs, writeout
// / writeenv / readout / get_ssp / get_percent_progress / finalize behave as
// the reference's. Every call returns false on failure and reports the reason
// through bhcInit::outputCallback; no exception leaves a bhc:: function.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/bhcb.h"
#include "../../../include/bhcb/bhc.hpp"
#include "env2d.h"

namespace bhc {

namespace {

constexpr double kPi = 3.14159265358979323846;

// Program state behind bhcParams::internal.
struct Internal {
    bhcInit init;
    std::string root;            // FileRoot of setup ("" after the defaults)
    int dim = 2;                 // 2, 3 (3-D) or 4 (Nx2D)
    bhcb_ctx *ctx = nullptr;
    bool blocking = true;
    std::thread worker;          // non-blocking run
    std::atomic<int> progress{100};
    std::atomic<bool> ok{true};
    std::string error;
    std::ofstream prt;           // FileRoot.prt when there is no prtCallback
};

Internal *state(const void *p) { return static_cast<Internal *>(const_cast<void *>(p)); }

void say(const Internal &in, const std::string &m)
{
    if(in.init.outputCallback) in.init.outputCallback(m.c_str());
    else std::printf("%s\n", m.c_str());
}

// PRT text: to prtCallback, else to FileRoot.prt (opened by setup), else
// stdout (PrintFileEmu, src/util/prtfileemu.hpp:30-60)
void prt(Internal &in, const std::string &m)
{
    if(in.init.prtCallback) in.init.prtCallback(m.c_str());
    else if(in.prt.is_open()) in.prt << m << std::flush;
    else std::printf("%s", m.c_str());
}

std::string last_error(bhcb_ctx *ctx)
{
    char b[512] = {0};
    uint32_t eb = 0, wb = 0;
    if(ctx) bhcb_last_error(ctx, b, sizeof b, &eb, &wb);
    return b;
}

void check(bhcb_ctx *ctx, int rc, const char *what)
{
    if(rc != BHCB_OK) throw std::runtime_error(std::string(what) + ": " + last_error(ctx));
}

template<typename T> T *alloc(size_t n)
{
    T *p = new T[n ? n : 1];
    std::memset(static_cast<void *>(p), 0, sizeof(T) * (n ? n : 1));
    return p;
}
template<typename T> void release(T *&p)
{
    delete[] p;
    p = nullptr;
}
template<typename T> void resize(T *&p, size_t n)
{
    release(p);
    p = alloc<T>(n);
}

// ------------------------------------------------------------ parameters
template<bool O3D> void alloc_params(bhcParams<O3D> &p)
{
    std::memset(p.Title, 0, sizeof p.Title);
    p.fT = 1e20;
    p.Bdry = alloc<BdryType>(1);
    p.bdinfo = alloc<BdryInfo<O3D>>(1);
    p.refl = alloc<ReflectionInfo>(1);
    p.ssp = alloc<SSPStructure>(1);
    p.ssp->z = alloc<real>(MaxSSP);
    p.ssp->rho = alloc<real>(MaxSSP);
    p.ssp->alphaR = alloc<real>(MaxSSP);
    p.ssp->alphaI = alloc<real>(MaxSSP);
    p.ssp->betaR = alloc<real>(MaxSSP);
    p.ssp->betaI = alloc<real>(MaxSSP);
    p.atten = alloc<AttenInfo>(1);
    p.Pos = alloc<Position>(1);
    p.Angles = alloc<AnglesStructure>(1);
    p.freqinfo = alloc<FreqInfo>(1);
    p.Beam = alloc<BeamStructure<O3D>>(1);
    p.sbp = alloc<SBPInfo>(1);
}

template<bool O3D> void free_params(bhcParams<O3D> &p)
{
    if(p.ssp) {
        release(p.ssp->z); release(p.ssp->rho); release(p.ssp->alphaR); release(p.ssp->alphaI);
        release(p.ssp->betaR); release(p.ssp->betaI); release(p.ssp->cMat); release(p.ssp->czMat);
        release(p.ssp->Seg.r); release(p.ssp->Seg.x); release(p.ssp->Seg.y); release(p.ssp->Seg.z);
    }
    if(p.bdinfo) {
        release(p.bdinfo->top.bd); release(p.bdinfo->bot.bd); release(p.bdinfo->bot.BotProv);
    }
    if(p.refl) { release(p.refl->top.r); release(p.refl->bot.r); }
    if(p.Pos) {
        release(p.Pos->Sx); release(p.Pos->Sy); release(p.Pos->Sz); release(p.Pos->Rr); release(p.Pos->Rz);
        release(p.Pos->theta); release(p.Pos->t_rcvr);
    }
    if(p.Angles) { release(p.Angles->alpha.angles); release(p.Angles->beta.angles); }
    if(p.freqinfo) release(p.freqinfo->freqVec);
    if(p.sbp) release(p.sbp->SrcBmPat);
    release(p.Bdry); release(p.bdinfo); release(p.refl); release(p.ssp); release(p.atten); release(p.Pos);
    release(p.Angles); release(p.freqinfo); release(p.Beam); release(p.sbp);
}

void set_title(char *dst, const char *src)
{
    std::memset(dst, 0, 80);
    if(src) std::strncpy(dst, src, 79);
}

// bhcParams<false> from a descriptor (file values, as the reference holds
// them after setup: ranges in km, angles in degrees, levels in dB)
void params_from_desc(bhcParams<false> &p, const bhcb_env_desc &d)
{
    set_title(p.Title, d.title);
    p.freqinfo->freq0 = d.freq0;
    p.freqinfo->Nfreq = 1;
    resize(p.freqinfo->freqVec, 1);
    p.freqinfo->freqVec[0] = d.freq0;
    BdryPtSmall *hb[2] = {&p.Bdry->Top, &p.Bdry->Bot};
    const double *hv[2] = {d.top_hs, d.bot_hs};
    std::memcpy(p.Bdry->Top.hs.Opt, d.top_opt, 6);
    std::memcpy(p.Bdry->Bot.hs.Opt, d.bot_opt, 6);
    p.Bdry->Top.hs.bc = d.top_opt[1];
    p.Bdry->Bot.hs.bc = d.bot_opt[0];
    for(int k = 0; k < 2; ++k) {
        hb[k]->hsx.zTemp = hv[k][0];
        hb[k]->hs.alphaR = hv[k][1];
        hb[k]->hs.betaR = hv[k][2];
        hb[k]->hs.rho = hv[k][3];
        hb[k]->hs.alphaI = hv[k][4];
        hb[k]->hs.betaI = hv[k][5];
        hb[k]->hsx.Mz = hv[k][6];
    }
    p.Bdry->Bot.hs.Depth = d.bot_depth;
    p.Bdry->Top.hs.Depth = d.nssp ? d.ssp_z[0] : 0.0;
    AttenInfo &a = *p.atten;
    a.t = d.fg[0]; a.Salinity = d.fg[1]; a.pH = d.fg[2]; a.z_bar = d.fg[3];
    a.NMedia = 1;
    a.NBioLayers = d.nbio;
    for(int i = 0; i < d.nbio && i < MaxBioLayers; ++i)
        a.bio[i] = bioStructure{d.bio[5 * i], d.bio[5 * i + 1], d.bio[5 * i + 2], d.bio[5 * i + 3], d.bio[5 * i + 4]};
    SSPStructure &s = *p.ssp;
    s.NPts = d.nssp;
    s.Nz = d.nssp;
    for(int i = 0; i < d.nssp; ++i) {
        s.z[i] = d.ssp_z[i]; s.alphaR[i] = d.ssp_alphaR[i]; s.betaR[i] = d.ssp_betaR[i];
        s.rho[i] = d.ssp_rho[i]; s.alphaI[i] = d.ssp_alphaI[i]; s.betaI[i] = d.ssp_betaI[i];
    }
    s.Type = d.top_opt[0];
    s.AttenUnit[0] = d.top_opt[2];
    s.AttenUnit[1] = d.top_opt[3];
    s.rangeInKm = true;
    s.dirty = true;
    s.Nr = d.nquad_r;
    if(d.nquad_r > 0) {
        resize(s.Seg.r, d.nquad_r);
        resize(s.cMat, (size_t)d.nquad_r * d.nssp);
        for(int i = 0; i < d.nquad_r; ++i) s.Seg.r[i] = d.quad_r_km[i];
        for(size_t i = 0; i < (size_t)d.nquad_r * d.nssp; ++i) s.cMat[i] = d.quad_c[i];
    }
    BdryInfoTopBot<false> *tb[2] = {&p.bdinfo->top, &p.bdinfo->bot};
    const int32_t nb[2] = {d.nati, d.nbty};
    const double *br[2] = {d.ati_r_km, d.bty_r_km}, *bz[2] = {d.ati_z, d.bty_z}, *bg[2] = {d.ati_geo, d.bty_geo};
    const char *bt[2] = {d.ati_type, d.bty_type};
    for(int k = 0; k < 2; ++k) {
        tb[k]->NPts = nb[k];   // 0: flat (no altimetry / bathymetry file)
        tb[k]->type[0] = bt[k][0];
        tb[k]->type[1] = bt[k][1];
        tb[k]->rangeInKm = true;
        tb[k]->dirty = true;
        resize(tb[k]->bd, nb[k]);
        for(int i = 0; i < nb[k]; ++i) {
            tb[k]->bd[i].x = vec2{br[k][i], bz[k][i]};
            if(bg[k]) {
                HSInfo &h = tb[k]->bd[i].hs;
                h.alphaR = bg[k][5 * i]; h.betaR = bg[k][5 * i + 1]; h.rho = bg[k][5 * i + 2];
                h.alphaI = bg[k][5 * i + 3]; h.betaI = bg[k][5 * i + 4];
            }
        }
    }
    ReflectionInfoTopBot *rt[2] = {&p.refl->top, &p.refl->bot};
    const int32_t nr[2] = {d.ntrc, d.nbrc};
    const double *rv[2] = {d.trc, d.brc};
    for(int k = 0; k < 2; ++k) {
        rt[k]->NPts = nr[k];
        rt[k]->inDegrees = true;
        resize(rt[k]->r, nr[k]);
        for(int i = 0; i < nr[k]; ++i) rt[k]->r[i] = ReflectionCoef{rv[k][3 * i], rv[k][3 * i + 1], rv[k][3 * i + 2]};
    }
    Position &P = *p.Pos;
    P.NSx = P.NSy = P.Ntheta = 1;
    resize(P.Sx, 1); resize(P.Sy, 1); resize(P.theta, 1); resize(P.t_rcvr, 1);
    P.t_rcvr[0] = vec2{1.0, 0.0};
    P.NSz = d.nsz; resize(P.Sz, d.nsz);
    for(int i = 0; i < d.nsz; ++i) P.Sz[i] = d.sz[i];
    P.NRz = d.nrz; resize(P.Rz, d.nrz);
    for(int i = 0; i < d.nrz; ++i) P.Rz[i] = d.rz[i];
    P.NRr = d.nrr; resize(P.Rr, d.nrr);
    for(int i = 0; i < d.nrr; ++i) P.Rr[i] = d.rr_km[i];
    P.RrInKm = true;
    P.SxSyInKm = true;
    P.NRz_per_range = d.run_type[4] == 'I' ? 1 : d.nrz;
    P.Delta_r = d.nrr >= 2 ? (d.rr_km[d.nrr - 1] - d.rr_km[d.nrr - 2]) : 0.0;
    AngleInfo &al = p.Angles->alpha;
    al.iSingle = d.isingle;
    al.inDegrees = true;
    if(d.nalpha > 0) {
        al.n = d.nalpha;
        resize(al.angles, std::max(d.nalpha, 2));
        for(int i = 0; i < std::max(d.nalpha, 2); ++i) al.angles[i] = d.alpha_deg[i];
    } else {
        // estimated count (src/module/rayangles.hpp:212-238): the fan the run
        // would trace, written out as explicit angles
        // (sub-tabulated in degrees as preprocessing does, so that the run
        // launches the same rays as from the estimate itself)
        const bhcb::EnvTables T = bhcb::preprocess(bhcb::env_from_desc(d), d.freq0);
        const int na = (int)T.alpha.size();
        std::vector<double> a = {d.alpha_deg[0], d.alpha_deg[1], -999.9};
        bhcb::subtab(a, na);
        a.resize(na);
        std::sort(a.begin(), a.end());
        al.n = na;
        resize(al.angles, std::max(na, 2));
        for(int i = 0; i < na; ++i) al.angles[i] = a[i];
    }
    al.d = al.n > 1 ? (al.angles[al.n - 1] - al.angles[0]) / (al.n - 1) : 0.0;
    BeamStructure<false> &B = *p.Beam;
    std::memcpy(B.RunType, d.run_type, 7);
    B.Type[0] = d.run_type[1];
    B.Type[1] = d.cerv_type[0];
    B.Type[2] = d.cerv_type[1];
    B.Type[3] = ' ';
    B.deltas = d.deltas;
    B.autoDeltas = d.deltas == 0.0;
    B.Box = vec2{d.box_r_km, d.box_z};
    B.rangeInKm = true;
    B.epsMultiplier = d.eps_mult;
    B.rLoop = d.rloop;
    B.Nimage = d.nimage;
    B.iBeamWindow = d.ibeam_window;
    B.Component = d.component;
    B.NBeams = al.n;
    SBPInfo &b = *p.sbp;
    b.SBPFlag = d.run_type[2];
    b.SBPIndB = true;
    b.NSBPPts = d.nsbp ? d.nsbp : 2;
    resize(b.SrcBmPat, 2 * (size_t)b.NSBPPts);
    if(d.nsbp) {
        for(int i = 0; i < 2 * d.nsbp; ++i) b.SrcBmPat[i] = d.sbp[i];
    } else {   // omnidirectional (src/module/sbp.hpp:43-53)
        b.SrcBmPat[0] = -180.0; b.SrcBmPat[1] = 0.0; b.SrcBmPat[2] = 180.0; b.SrcBmPat[3] = 0.0;
    }
}

// The descriptor of bhcParams<false> (with the arrays it points into), unit
// flags applied: ranges back to km, angles to degrees, levels to dB.
struct DescOf {
    bhcb_env_desc d;
    std::string title;
    std::vector<double> bio, ssp_z, aR, bR, rho, aI, bI, ati_r, ati_z, ati_g, bty_r, bty_z, bty_g, sbp, rr, al;
    std::vector<double> qr, qc, brc, trc;
    std::vector<float> sz, rz;

    explicit DescOf(const bhcParams<false> &p)
    {
        std::memset(&d, 0, sizeof d);
        title = std::string(p.Title, strnlen(p.Title, 80));
        d.title = title.c_str();
        d.freq0 = p.freqinfo->freq0;
        std::memcpy(d.top_opt, p.Bdry->Top.hs.Opt, 6);
        std::memcpy(d.bot_opt, p.Bdry->Bot.hs.Opt, 6);
        d.top_opt[1] = p.Bdry->Top.hs.bc ? p.Bdry->Top.hs.bc : d.top_opt[1];
        d.bot_opt[0] = p.Bdry->Bot.hs.bc ? p.Bdry->Bot.hs.bc : d.bot_opt[0];
        d.fg[0] = p.atten->t; d.fg[1] = p.atten->Salinity; d.fg[2] = p.atten->pH; d.fg[3] = p.atten->z_bar;
        for(int i = 0; i < p.atten->NBioLayers && i < MaxBioLayers; ++i) {
            const bioStructure &b = p.atten->bio[i];
            bio.insert(bio.end(), {b.z1, b.z2, b.f0, b.q, b.a0});
        }
        d.nbio = (int32_t)(bio.size() / 5);
        d.bio = bio.data();
        const BdryPtSmall *hb[2] = {&p.Bdry->Top, &p.Bdry->Bot};
        double *hv[2] = {d.top_hs, d.bot_hs};
        for(int k = 0; k < 2; ++k) {
            hv[k][0] = hb[k]->hsx.zTemp; hv[k][1] = hb[k]->hs.alphaR; hv[k][2] = hb[k]->hs.betaR;
            hv[k][3] = hb[k]->hs.rho; hv[k][4] = hb[k]->hs.alphaI; hv[k][5] = hb[k]->hs.betaI;
            hv[k][6] = hb[k]->hsx.Mz;
        }
        const SSPStructure &s = *p.ssp;
        if(s.NPts < 2 || s.NPts > MaxSSP) throw std::invalid_argument("ssp->NPts must be in 2..MaxSSP");
        ssp_z.assign(s.z, s.z + s.NPts); aR.assign(s.alphaR, s.alphaR + s.NPts); bR.assign(s.betaR, s.betaR + s.NPts);
        rho.assign(s.rho, s.rho + s.NPts); aI.assign(s.alphaI, s.alphaI + s.NPts); bI.assign(s.betaI, s.betaI + s.NPts);
        d.nssp = s.NPts;
        d.ssp_z = ssp_z.data(); d.ssp_alphaR = aR.data(); d.ssp_betaR = bR.data(); d.ssp_rho = rho.data();
        d.ssp_alphaI = aI.data(); d.ssp_betaI = bI.data();
        if(s.Type) d.top_opt[0] = s.Type;
        d.bot_depth = p.Bdry->Bot.hs.Depth;
        if(s.Nr > 0 && s.Seg.r && s.cMat) {
            for(int i = 0; i < s.Nr; ++i) qr.push_back(s.rangeInKm ? s.Seg.r[i] : s.Seg.r[i] / 1000.0);
            qc.assign(s.cMat, s.cMat + (size_t)s.Nr * s.NPts);
            d.nquad_r = s.Nr;
            d.quad_r_km = qr.data();
            d.quad_c = qc.data();
        }
        const BdryInfoTopBot<false> *tb[2] = {&p.bdinfo->top, &p.bdinfo->bot};
        std::vector<double> *R[2] = {&ati_r, &bty_r}, *Z[2] = {&ati_z, &bty_z}, *G[2] = {&ati_g, &bty_g};
        for(int k = 0; k < 2; ++k) {
            for(int i = 0; i < tb[k]->NPts; ++i) {
                const BdryPtFull<false> &b = tb[k]->bd[i];
                R[k]->push_back(tb[k]->rangeInKm ? b.x.x : b.x.x / 1000.0);
                Z[k]->push_back(b.x.y);
                G[k]->insert(G[k]->end(), {b.hs.alphaR, b.hs.betaR, b.hs.rho, b.hs.alphaI, b.hs.betaI});
            }
        }
        d.ati_type[0] = p.bdinfo->top.type[0]; d.ati_type[1] = p.bdinfo->top.type[1];
        d.bty_type[0] = p.bdinfo->bot.type[0]; d.bty_type[1] = p.bdinfo->bot.type[1];
        d.nati = p.bdinfo->top.NPts; d.nbty = p.bdinfo->bot.NPts;
        d.ati_r_km = ati_r.data(); d.ati_z = ati_z.data(); d.ati_geo = ati_g.data();
        d.bty_r_km = bty_r.data(); d.bty_z = bty_z.data(); d.bty_geo = bty_g.data();
        d.top_opt[4] = d.nati ? '~' : (d.top_opt[4] == '~' || d.top_opt[4] == '*' ? ' ' : d.top_opt[4]);
        d.bot_opt[1] = d.nbty ? '~' : (d.bot_opt[1] == '~' || d.bot_opt[1] == '*' ? ' ' : d.bot_opt[1]);
        const ReflectionInfoTopBot *rt[2] = {&p.refl->top, &p.refl->bot};
        std::vector<double> *RV[2] = {&trc, &brc};
        for(int k = 0; k < 2; ++k)
            for(int i = 0; i < rt[k]->NPts; ++i) {
                const ReflectionCoef &c = rt[k]->r[i];
                RV[k]->insert(RV[k]->end(), {c.theta, c.r, rt[k]->inDegrees ? c.phi : c.phi * 180.0 / kPi});
            }
        d.ntrc = p.refl->top.NPts; d.nbrc = p.refl->bot.NPts;
        d.trc = trc.data(); d.brc = brc.data();
        const Position &P = *p.Pos;
        sz.assign(P.Sz, P.Sz + P.NSz);
        rz.assign(P.Rz, P.Rz + P.NRz);
        for(int i = 0; i < P.NRr; ++i) rr.push_back(P.RrInKm ? P.Rr[i] : P.Rr[i] / 1000.0);
        d.nsz = P.NSz; d.nrz = P.NRz; d.nrr = P.NRr;
        d.sz = sz.data(); d.rz = rz.data(); d.rr_km = rr.data();
        const AngleInfo &a = p.Angles->alpha;
        for(int i = 0; i < std::max(a.n, 2); ++i) al.push_back(a.inDegrees ? a.angles[i] : a.angles[i] * 180.0 / kPi);
        d.nalpha = a.n;
        d.isingle = a.iSingle;
        d.alpha_deg = al.data();
        if(a.iSingle > 0) d.top_opt[5] = 'I';
        const BeamStructure<false> &B = *p.Beam;
        std::memcpy(d.run_type, B.RunType, 7);
        d.cerv_type[0] = B.Type[1];
        d.cerv_type[1] = B.Type[2];
        d.deltas = B.deltas;
        d.box_r_km = B.rangeInKm ? B.Box.x : B.Box.x / 1000.0;
        d.box_z = B.Box.y;
        d.eps_mult = B.epsMultiplier;
        d.rloop = B.rLoop;
        d.nimage = B.Nimage;
        d.ibeam_window = B.iBeamWindow;
        d.component = B.Component;
        const SBPInfo &b = *p.sbp;
        if(b.SBPFlag == '*') {
            for(int i = 0; i < b.NSBPPts; ++i) {
                sbp.push_back(b.SrcBmPat[2 * i]);
                const double lv = b.SrcBmPat[2 * i + 1];
                sbp.push_back(b.SBPIndB ? lv : 20.0 * std::log10(lv));
            }
            d.nsbp = b.NSBPPts;
            d.run_type[2] = '*';
        }
        d.sbp = sbp.data();
    }
};

// The modules' defaults (src/module/*.hpp Default(), FileRoot == nullptr):
// Munk-free isovelocity 1500 m/s over a rigid bottom at 5000 m, source at
// 567.8 m, 11 receiver depths 0..5000 m, 10 ranges 5..50 km, 50 Hz, coherent
// TL with geometric hat beams over -20..20 degrees (count estimated).
void default_desc_2d(std::vector<double> &z, std::vector<double> &c, std::vector<double> &one,
                     std::vector<double> &zero, std::vector<float> &sz, std::vector<float> &rz,
                     std::vector<double> &rr, std::vector<double> &al, bhcb_env_desc &d)
{
    std::memset(&d, 0, sizeof d);
    d.title = "no env file";
    d.freq0 = 50.0;
    std::memcpy(d.top_opt, "CVW - ", 6);
    std::memcpy(d.bot_opt, "R-    ", 6);
    d.fg[0] = 20.0; d.fg[1] = 35.0; d.fg[2] = 8.0; d.fg[3] = 0.0;
    z = {0.0, 5000.0};
    c = {1500.0, 1500.0};
    one = {1.0, 1.0};
    zero = {0.0, 0.0};
    d.nssp = 2;
    d.ssp_z = z.data(); d.ssp_alphaR = c.data(); d.ssp_betaR = zero.data(); d.ssp_rho = one.data();
    d.ssp_alphaI = zero.data(); d.ssp_betaI = zero.data();
    d.bot_depth = 5000.0;
    d.ati_type[0] = d.bty_type[0] = 'L';
    d.ati_type[1] = d.bty_type[1] = 'S';
    sz = {567.8f};
    rz.clear();
    for(int i = 0; i < 11; ++i) rz.push_back(500.0f * (float)i);
    rr.clear();
    for(int i = 0; i < 10; ++i) rr.push_back(5.0 * (i + 1));
    al = {-20.0, 20.0};
    d.nsz = 1; d.nrz = 11; d.nrr = 10; d.nalpha = 0;
    d.sz = sz.data(); d.rz = rz.data(); d.rr_km = rr.data(); d.alpha_deg = al.data();
    std::memcpy(d.run_type, "CG RR  ", 7);
    d.cerv_type[0] = ' ';
    d.cerv_type[1] = 'S';
    d.box_r_km = 101.0;
    d.box_z = 6000.0;
    d.eps_mult = 1.0;
    d.rloop = 1.0;
    d.nimage = 1;
    d.ibeam_window = 4;
    d.component = 'P';
}

bhcb_ctx *open_ctx(Internal &in)
{
    if(in.ctx) return in.ctx;
    bhcb_init bi{};
    bi.gpu_index = in.init.gpuIndex;
    const char *prec = std::getenv("BHCB_PRECISION");
    bi.precision = (prec && std::strcmp(prec, "mixed") == 0) ? BHCB_PREC_MIXED : BHCB_PREC_FP64;
    bi.max_memory = in.init.maxMemory;
    bi.share_trajectory = 1;
    bi.output_callback = in.init.outputCallback;
    if(bhcb_open(&bi, &in.ctx) != BHCB_OK) {
        in.ctx = nullptr;
        throw std::runtime_error("no usable CUDA device (gpuIndex " + std::to_string(in.init.gpuIndex) + ")");
    }
    return in.ctx;
}

template<bool O3D> Internal &internal_of(const bhcParams<O3D> &p)
{
    if(!p.internal) throw std::runtime_error("bhc::setup has not been called on these parameters");
    return *state(p.internal);
}

// ---------------------------------------------------------------- outputs
template<bool O3D, bool R3D> void free_outputs(bhcOutputs<O3D, R3D> &o)
{
    delete[] o.uAllSources;
    o.uAllSources = nullptr;
    if(o.arrinfo) {
        delete[] o.arrinfo->Arr; delete[] o.arrinfo->NArr; delete[] o.arrinfo->MaxNPerSource;
        delete o.arrinfo;
        o.arrinfo = nullptr;
    }
    if(o.eigen) {
        delete[] o.eigen->hits;
        delete o.eigen;
        o.eigen = nullptr;
    }
    if(o.rayinfo) {
        for(int i = 0; i < o.rayinfo->NRays; ++i) delete[] o.rayinfo->results[i].ray;
        delete[] o.rayinfo->results;
        delete o.rayinfo;
        o.rayinfo = nullptr;
    }
}

template<bool O3D, bool R3D> void collect(Internal &in, bhcOutputs<O3D, R3D> &o, char run0)
{
    bhcb_ctx *ctx = in.ctx;
    free_outputs(o);
    o.arrinfo = new ArrInfo{};
    o.eigen = new EigenInfo{};
    o.rayinfo = new RayInfo<O3D, R3D>{};
    if(run0 == 'C' || run0 == 'S' || run0 == 'I') {
        size_t n = 0;
        if(in.dim == 2) {
            int32_t nf = 0, nsz = 0, nrz = 0, nrr = 0;
            check(ctx, bhcb_field_shape(ctx, 0, &nf, &nsz, &nrz, &nrr), "field shape");
            n = (size_t)nsz * nrz * nrr;
        } else {
            int32_t dims[6] = {0};
            check(ctx, bhcb_field_shape3d(ctx, 0, dims), "field shape");
            n = 1;
            for(int k = 0; k < 6; ++k) n *= (size_t)dims[k];
        }
        o.uAllSources = new cpxf[n];
        check(ctx, bhcb_copy_field(ctx, 0, 0, o.uAllSources, n * sizeof(cpxf)), "copy field");
    }
    const bool combined = run0 == 'V' || run0 == 'v';   // arrivals and eigen hits in one run
    if(run0 == 'A' || run0 == 'a' || combined) {
        int32_t nsz = 0, nrz = 0, nrr = 0, mx = 0;
        check(ctx, bhcb_arrivals_shape(ctx, 0, 0, &nsz, &nrz, &nrr, &mx), "arrivals shape");
        const size_t cells = (size_t)nsz * nrz * nrr;
        o.arrinfo->NArr = new int32_t[cells];
        o.arrinfo->Arr = new Arrival[cells * mx];
        o.arrinfo->MaxNArr = mx;
        o.arrinfo->AllowMerging = in.init.numThreads == 1;
        // MaxNPerSource is per source (NSx * NSy * NSz); in 3-D the shape's
        // leading count also spans the bearings, whose cells follow their
        // source's in the [isz][isx][isy][itheta][iz][ir] layout
        int32_t nsrc = nsz;
        if(in.dim != 2) {
            int32_t d[6] = {0};
            check(ctx, bhcb_field_shape3d(ctx, 0, d), "field shape");
            nsrc = d[0] * d[1] * d[2];
        }
        o.arrinfo->MaxNPerSource = new int32_t[nsrc > 0 ? nsrc : 1];
        std::vector<bhcb_arrival> a(cells * mx);
        check(ctx, bhcb_copy_arrivals(ctx, 0, 0, o.arrinfo->NArr, cells * sizeof(int32_t), a.data(),
                                      a.size() * sizeof(bhcb_arrival)), "copy arrivals");
        for(size_t i = 0; i < a.size(); ++i) {
            Arrival &r = o.arrinfo->Arr[i];
            r.NTopBnc = a[i].ntop; r.NBotBnc = a[i].nbot;
            r.SrcDeclAngle = a[i].src_decl; r.SrcAzimAngle = a[i].src_azim;
            r.RcvrDeclAngle = a[i].rcvr_decl; r.RcvrAzimAngle = a[i].rcvr_azim;
            r.a = a[i].a; r.Phase = a[i].phase;
            r.delay = cpxf(a[i].delay_re, a[i].delay_im);
        }
        const size_t per = cells / (nsrc ? nsrc : 1);
        for(int s = 0; s < nsrc; ++s) {
            int32_t m = 0;
            for(size_t i = 0; i < per; ++i) m = std::max(m, o.arrinfo->NArr[s * per + i]);
            o.arrinfo->MaxNPerSource[s] = m;
        }
    }
    if(run0 == 'E' || combined) {
        int64_t nh = 0;
        check(ctx, bhcb_eigen_hits(ctx, 0, 0, nullptr, 0, &nh), "eigen hits");
        std::vector<bhcb_eigen_hit> h((size_t)nh);
        check(ctx, bhcb_eigen_hits(ctx, 0, 0, h.data(), nh, &nh), "eigen hits");
        o.eigen->neigen = (int32_t)nh;
        o.eigen->memsize = (int32_t)nh;
        o.eigen->hits = new EigenHit[nh ? nh : 1];
        for(int64_t i = 0; i < nh; ++i)
            o.eigen->hits[i] = EigenHit{h[i].is, h[i].itheta, h[i].ir, h[i].iz, h[i].isx, h[i].isy, h[i].isz,
                                        h[i].ialpha, h[i].ibeta};
    }
    if(run0 == 'R' || run0 == 'E' || combined) {   // trajectories: rays of a ray run, hit rays of an eigen run
        int64_t nrays = 0, npts = 0;
        if(bhcb_rays_shape(ctx, 0, 0, &nrays, &npts) == BHCB_OK && nrays > 0) {
            // 2 doubles (r, z) per point from a 2-D context, 3 (x, y, z) from a
            // 3-D one; Nx2D rays (R3D false) become (distance from the source, z)
            const int dsrc = in.dim == 2 ? 2 : 3;
            std::vector<int32_t> np((size_t)nrays), bnc(2 * (size_t)nrays);
            std::vector<double> alpha((size_t)nrays), pts((size_t)npts * dsrc);
            check(ctx, bhcb_copy_rays(ctx, 0, 0, np.data(), bnc.data(), alpha.data(), pts.data(),
                                      pts.size() * sizeof(double)), "copy rays");
            o.rayinfo->NRays = (int32_t)nrays;
            o.rayinfo->results = new RayResult<O3D, R3D>[nrays];
            size_t off = 0;
            for(int64_t r = 0; r < nrays; ++r) {
                RayResult<O3D, R3D> &res = o.rayinfo->results[r];
                res.Nsteps = np[r];
                res.SrcDeclAngle = alpha[r];
                res.ray = new rayPt<R3D>[np[r] ? np[r] : 1]();
                const double *p0 = &pts[off * dsrc];
                for(int k = 0; k < np[r]; ++k, ++off) {
                    rayPt<R3D> &pt = res.ray[k];
                    const double *q = &pts[off * dsrc];
                    if constexpr(R3D) {
                        pt.x = vec3{q[0], q[1], q[2]};
                    } else if(dsrc == 3) {
                        pt.x = vec2{std::hypot(q[0] - p0[0], q[1] - p0[1]), q[2]};
                    } else {
                        pt.x = vec2{q[0], q[1]};
                    }
                    pt.NumTopBnc = k + 1 == np[r] ? bnc[2 * r] : 0;
                    pt.NumBotBnc = k + 1 == np[r] ? bnc[2 * r + 1] : 0;
                }
            }
        }
    }
}

// The run itself (blocking or on the worker thread).
template<bool O3D, bool R3D> void run_now(bhcParams<O3D> &p, bhcOutputs<O3D, R3D> &o)
{
    Internal &in = internal_of(p);
    bhcb_ctx *ctx = open_ctx(in);
    in.progress = 0;
    char run0 = 'C';
    if(in.dim == 2) {
        if constexpr(!O3D) {
            DescOf d(p);
            run0 = d.d.run_type[0];
            check(ctx, bhcb_clear(ctx), "clear");
            check(ctx, bhcb_add_env_desc(ctx, &d.d, nullptr), "environment");
        }
    } else {
        if(in.root.empty()) throw std::runtime_error("3-D and Nx2D runs read FileRoot's files (setup with FileRoot)");
        check(ctx, bhcb_setup3d(ctx, in.root.c_str()), "3-D setup");
        run0 = p.Beam->RunType[0];
    }
    if(run0 == 'A' || run0 == 'a' || run0 == 'V' || run0 == 'v') {
        // merging as the reference's Arr mode decides it: only single-threaded
        // runs merge (AllowMerging, src/mode/arr.hpp:78); MaxNArr from memory
        check(ctx, bhcb_set_arrival_options(ctx, 0, in.init.numThreads == 1 ? 1 : 0), "arrival options");
    }
    in.progress = 10;
    check(ctx, bhcb_run(ctx), "run");
    in.progress = 90;
    collect(in, o, run0);
    in.progress = 100;
}

std::string fmt(double v)
{
    char b[64];
    std::snprintf(b, sizeof b, "%.17g", v);
    return b;
}

// 2-D .env (+ .bty, .ati, .sbp, .brc, .trc, quad .ssp) from a descriptor, in
// the grammar of src/api.cpp:253-277 (module Write() order)
void write_env_files(const bhcb_env_desc &d, const std::string &root)
{
    std::ofstream f(root + ".env");
    if(!f) throw std::runtime_error("cannot write " + root + ".env");
    f << "'" << (d.title ? d.title : "") << "' ! TITLE\n";
    f << fmt(d.freq0) << " ! FREQ (Hz)\n1 ! NMEDIA\n";
    f << "'" << std::string(d.top_opt, 6) << "' ! SSP, top bc, atten units, add vol atten, altimetry, single beam\n";
    if(d.top_opt[3] == 'F') f << fmt(d.fg[0]) << " " << fmt(d.fg[1]) << " " << fmt(d.fg[2]) << " " << fmt(d.fg[3]) << "\n";
    if(d.top_opt[3] == 'B') {
        f << d.nbio << "\n";
        for(int i = 0; i < d.nbio; ++i)
            f << fmt(d.bio[5 * i]) << " " << fmt(d.bio[5 * i + 1]) << " " << fmt(d.bio[5 * i + 2]) << " "
              << fmt(d.bio[5 * i + 3]) << " " << fmt(d.bio[5 * i + 4]) << "\n";
    }
    auto hs = [&](const double *v, char bc) {
        if(bc == 'A') {
            f << fmt(v[0]);
            for(int k = 1; k < 6; ++k) f << " " << fmt(v[k]);
            f << " /\n";
        } else if(bc == 'G') {
            f << fmt(v[0]) << " " << fmt(v[6]) << " /\n";
        }
    };
    hs(d.top_hs, d.top_opt[1]);
    f << d.nssp << " 0.0 " << fmt(d.bot_depth) << "\n";
    for(int i = 0; i < d.nssp; ++i)
        f << fmt(d.ssp_z[i]) << " " << fmt(d.ssp_alphaR[i]) << " " << fmt(d.ssp_betaR[i]) << " " << fmt(d.ssp_rho[i])
          << " " << fmt(d.ssp_alphaI[i]) << " " << fmt(d.ssp_betaI[i]) << " /\n";
    std::string bo(d.bot_opt, 6);
    bo.erase(bo.find_last_not_of(' ') + 1);
    f << "'" << bo << "' 0.0\n";
    hs(d.bot_hs, d.bot_opt[0]);
    auto vecf = [&](int n, const float *v) {
        f << n << "\n";
        for(int i = 0; i < n; ++i) f << fmt(v[i]) << (i + 1 < n ? " " : " /\n");
    };
    auto vecd = [&](int n, const double *v) {
        f << n << "\n";
        for(int i = 0; i < n; ++i) f << fmt(v[i]) << (i + 1 < n ? " " : " /\n");
    };
    vecf(d.nsz, d.sz);
    vecf(d.nrz, d.rz);
    vecd(d.nrr, d.rr_km);
    f << "'" << std::string(d.run_type, 7) << "'\n";
    if(d.top_opt[5] == 'I') f << d.nalpha << " " << d.isingle << "\n";
    else f << d.nalpha << "\n";
    const int na = d.nalpha ? d.nalpha : 2;
    for(int i = 0; i < na; ++i) f << fmt(d.alpha_deg[i]) << (i + 1 < na ? " " : " /\n");
    f << fmt(d.deltas) << " " << fmt(d.box_z) << " " << fmt(d.box_r_km) << "\n";
    if(d.run_type[0] != 'R' && (d.run_type[1] == 'C' || d.run_type[1] == 'R')) {
        f << "'" << d.cerv_type[0] << d.cerv_type[1] << "' " << fmt(d.eps_mult) << " " << fmt(d.rloop) << "\n";
        f << d.nimage << " " << d.ibeam_window << " '" << d.component << "'\n";
    }
    auto bdry = [&](const char *ext, const char type[2], int n, const double *r, const double *z, const double *g) {
        std::ofstream b(root + ext);
        b << "'" << type[0] << type[1] << "'\n" << n << "\n";
        for(int i = 0; i < n; ++i) {
            b << fmt(r[i]) << " " << fmt(z[i]);
            if(type[1] == 'L' && g)
                for(int k = 0; k < 5; ++k) b << " " << fmt(g[5 * i + k]);
            b << "\n";
        }
    };
    if(d.nati) bdry(".ati", d.ati_type, d.nati, d.ati_r_km, d.ati_z, d.ati_geo);
    if(d.nbty) bdry(".bty", d.bty_type, d.nbty, d.bty_r_km, d.bty_z, d.bty_geo);
    if(d.nsbp) {
        std::ofstream s(root + ".sbp");
        s << d.nsbp << "\n";
        for(int i = 0; i < d.nsbp; ++i) s << fmt(d.sbp[2 * i]) << " " << fmt(d.sbp[2 * i + 1]) << "\n";
    }
    auto refl = [&](const char *ext, int n, const double *t) {
        std::ofstream r(root + ext);
        r << n << "\n";
        for(int i = 0; i < n; ++i) r << fmt(t[3 * i]) << " " << fmt(t[3 * i + 1]) << " " << fmt(t[3 * i + 2]) << "\n";
    };
    if(d.bot_opt[0] == 'F') refl(".brc", d.nbrc, d.brc);
    if(d.top_opt[1] == 'F') refl(".trc", d.ntrc, d.trc);
    if(d.top_opt[0] == 'Q' && d.nquad_r) {
        std::ofstream q(root + ".ssp");
        q << d.nquad_r << "\n";
        for(int i = 0; i < d.nquad_r; ++i) q << fmt(d.quad_r_km[i]) << (i + 1 < d.nquad_r ? " " : "\n");
        for(int iz = 0; iz < d.nssp; ++iz)
            for(int ir = 0; ir < d.nquad_r; ++ir)
                q << fmt(d.quad_c[(size_t)iz * d.nquad_r + ir]) << (ir + 1 < d.nquad_r ? " " : "\n");
    }
}

// Fixed-length records of a .shd file (direct access; the first word of
// record 0 is the record length in 4-byte words, src/mode/tl.cpp:38-101)
struct ShdReader {
    std::ifstream f;
    size_t lrecl = 0;
    explicit ShdReader(const std::string &p) : f(p, std::ios::binary)
    {
        int32_t lw = 0;
        if(!f.read(reinterpret_cast<char *>(&lw), 4) || lw < 21) throw std::runtime_error("cannot read " + p);
        lrecl = (size_t)lw * 4;
    }
    std::vector<char> rec(size_t k)
    {
        std::vector<char> b(lrecl);
        f.clear();
        f.seekg((std::streamoff)(k * lrecl));
        if(!f.read(b.data(), (std::streamsize)lrecl)) throw std::runtime_error("truncated .shd file");
        return b;
    }
};

// List-directed text (the reference's LDIFile as its output readers use it):
// list() starts a read statement at the next line; values are separated by
// blanks or commas, strings may be quoted, and a statement continues onto
// the following lines until it has its values.
struct ListIn {
    std::vector<std::string> lines;
    size_t li = 0, pos = 0;
    bool started = false;
    explicit ListIn(const std::string &p)
    {
        std::ifstream f(p);
        if(!f.good()) throw std::runtime_error("cannot open " + p);
        std::string l;
        while(std::getline(f, l)) lines.push_back(l);
    }
    void list()
    {
        if(started) { ++li; pos = 0; }
        started = true;
    }
    bool eof()
    {
        size_t k = started ? li + 1 : li;
        for(; k < lines.size(); ++k)
            if(lines[k].find_first_not_of(" \t\r,") != std::string::npos) return false;
        return true;
    }
    std::string token()
    {
        for(;;) {
            if(li >= lines.size()) throw std::runtime_error("end of file in a list-directed read");
            const std::string &l = lines[li];
            while(pos < l.size() && (l[pos] == ' ' || l[pos] == '\t' || l[pos] == '\r' || l[pos] == ',')) ++pos;
            if(pos >= l.size()) { ++li; pos = 0; continue; }
            if(l[pos] == '\'' || l[pos] == '"') {
                const char q = l[pos];
                const size_t e = l.find(q, pos + 1);
                std::string t = l.substr(pos + 1, (e == std::string::npos ? l.size() : e) - pos - 1);
                pos = e == std::string::npos ? l.size() : e + 1;
                return t;
            }
            size_t e = pos;
            while(e < l.size() && l[e] != ' ' && l[e] != '\t' && l[e] != '\r' && l[e] != ',') ++e;
            std::string t = l.substr(pos, e - pos);
            pos = e;
            return t;
        }
    }
    double real() { return std::stod(token()); }
    int32_t integer() { return (int32_t)std::lround(std::stod(token())); }
};

// Fortran sequential unformatted records ([int32 n][n bytes][int32 n], the
// reference's UnformattedIFile): rec() moves to the next record, get() reads
// the record's values in order.
struct SeqIn {
    std::vector<char> b;
    size_t next = 0, cur = 0, end = 0;
    explicit SeqIn(const std::string &p)
    {
        std::ifstream f(p, std::ios::binary);
        if(!f.good()) throw std::runtime_error("cannot open " + p);
        b.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    }
    void rec()
    {
        int32_t n = 0;
        if(next + 4 > b.size()) throw std::runtime_error("end of file in an unformatted read");
        std::memcpy(&n, b.data() + next, 4);
        if(n < 0 || next + 8 + (size_t)n > b.size()) throw std::runtime_error("bad record in an unformatted file");
        cur = next + 4;
        end = cur + (size_t)n;
        next = end + 4;
    }
    template<typename T> T get()
    {
        T v;
        if(cur + sizeof(T) > end) throw std::runtime_error("record too short in an unformatted file");
        std::memcpy(&v, b.data() + cur, sizeof(T));
        cur += sizeof(T);
        return v;
    }
};

// ReadOutArrivals (src/mode/arr.cpp:275-428): header (dimension, frequency,
// source and receiver coordinates), then per source its largest arrival
// count and per receiver the count and the records. MaxNArr is the largest
// count in the file within what the arrival memory of maxMemory holds
// (src/mode/arr.hpp:74-104); counts above it are cut, with a warning.
template<bool O3D, bool R3D> void read_arrivals(Internal &in, bhcParams<O3D> &params, bhcOutputs<O3D, R3D> &outputs,
                                                const std::string &path, bool ascii)
{
    std::unique_ptr<ListIn> A;
    std::unique_ptr<SeqIn> Bf;
    if(ascii) A.reset(new ListIn(path)); else Bf.reset(new SeqIn(path));
    auto beginv = [&]() { if(ascii) A->list(); else Bf->rec(); };
    auto rd_f = [&]() -> double { return ascii ? A->real() : (double)Bf->get<float>(); };
    auto rd_d = [&]() -> double { return ascii ? A->real() : Bf->get<double>(); };
    auto rd_i = [&]() -> int32_t { return ascii ? A->integer() : Bf->get<int32_t>(); };
    std::string dim;
    if(ascii) {
        A->list();
        dim = "'" + A->token() + "'";
    } else {
        Bf->rec();
        char t[4];
        for(char &c : t) c = Bf->get<char>();
        dim.assign(t, 4);
    }
    if(dim != (O3D ? "'3D'" : "'2D'"))
        throw std::runtime_error(std::string("incorrect dimensionality in arrivals file, must be ") +
                                 (O3D ? "'3D'" : "'2D'") + ", got " + dim);
    beginv();
    params.freqinfo->freq0 = (float)rd_f();
    Position &P = *params.Pos;
    auto rd_array_d = [&](double *&v, int32_t &n) {
        beginv();
        n = rd_i();
        if(n < 1) throw std::runtime_error("bad coordinate count in arrivals file");
        resize(v, (size_t)n);
        for(int32_t i = 0; i < n; ++i) v[i] = rd_d();
    };
    auto rd_array_f = [&](float *&v, int32_t &n) {
        beginv();
        n = rd_i();
        if(n < 1) throw std::runtime_error("bad coordinate count in arrivals file");
        resize(v, (size_t)n);
        for(int32_t i = 0; i < n; ++i) v[i] = (float)rd_f();
    };
    if constexpr(O3D) {
        rd_array_d(P.Sx, P.NSx);
        rd_array_d(P.Sy, P.NSy);
    } else {
        P.NSx = P.NSy = 1;
    }
    rd_array_f(P.Sz, P.NSz);
    rd_array_f(P.Rz, P.NRz);
    rd_array_d(P.Rr, P.NRr);
    if constexpr(O3D) {
        rd_array_d(P.theta, P.Ntheta);
    } else {
        P.Ntheta = 1;
    }
    if(params.Beam->RunType[4] == 'I')
        throw std::runtime_error("arrivals readout (and writeout) is not compatible with an irregular grid");
    P.NRz_per_range = P.NRz;
    P.RrInKm = false;
    const size_t nsrc = (size_t)P.NSx * P.NSy * P.NSz;
    const size_t per_src = (size_t)P.Ntheta * P.NRz * P.NRr;
    const size_t cells = nsrc * per_src;
    // every record first (the arrays are sized by the largest count)
    std::vector<int32_t> narr(cells, 0), maxn(nsrc, 0);
    std::vector<std::vector<Arrival>> recs(cells);
    const double DegRad = kPi / 180.0;
    for(int32_t isz = 0; isz < P.NSz; ++isz)
        for(int32_t isx = 0; isx < P.NSx; ++isx)
            for(int32_t isy = 0; isy < P.NSy; ++isy) {
                const size_t src = ((size_t)isz * P.NSx + isx) * P.NSy + isy;
                beginv();
                maxn[src] = rd_i();
                for(size_t k = 0; k < per_src; ++k) {
                    // GetFieldAddr order: [isz][isx][isy][itheta][iz][ir]
                    const size_t cell = src * per_src + k;
                    beginv();
                    const int32_t n = rd_i();
                    if(n < 0) throw std::runtime_error("negative arrival count in arrivals file");
                    narr[cell] = n;
                    recs[cell].resize((size_t)n);
                    for(int32_t a = 0; a < n; ++a) {
                        Arrival &R = recs[cell][a];
                        beginv();
                        R.a = (float)rd_f();
                        R.Phase = (float)(DegRad * (ascii ? A->real() : (double)Bf->get<float>()));
                        const float d1 = (float)rd_f(), d2 = (float)rd_f();
                        R.delay = cpxf(d1, d2);
                        R.SrcDeclAngle = (float)rd_f();
                        R.SrcAzimAngle = O3D ? (float)rd_f() : 0.f;
                        R.RcvrDeclAngle = (float)rd_f();
                        R.RcvrAzimAngle = O3D ? (float)rd_f() : 0.f;
                        if(ascii) {
                            R.NTopBnc = A->integer();
                            R.NBotBnc = A->integer();
                        } else {
                            R.NTopBnc = (int32_t)Bf->get<float>();
                            R.NBotBnc = (int32_t)Bf->get<float>();
                        }
                    }
                }
            }
    int64_t mem = (int64_t)in.init.maxMemory - (int64_t)(cells * sizeof(int32_t)) - (int64_t)(nsrc * sizeof(int32_t)) - 96;
    mem = std::max<int64_t>(mem, 0);
    const int64_t fit = mem / (int64_t)(cells * sizeof(Arrival));
    if(fit == 0) throw std::runtime_error("insufficient memory to allocate arrivals");
    int32_t most = 1;
    for(int32_t n : narr) most = std::max(most, n);
    const int32_t mx = (int32_t)std::min<int64_t>(most, std::min<int64_t>(fit, 0x7fffffff));
    free_outputs(outputs);
    outputs.arrinfo = new ArrInfo{};
    outputs.eigen = new EigenInfo{};
    outputs.rayinfo = new RayInfo<O3D, R3D>{};
    ArrInfo &I = *outputs.arrinfo;
    I.MaxNArr = mx;
    I.AllowMerging = in.init.numThreads == 1;
    I.NArr = new int32_t[cells];
    I.Arr = new Arrival[cells * (size_t)mx]();
    I.MaxNPerSource = new int32_t[nsrc];
    for(size_t s2 = 0; s2 < nsrc; ++s2) I.MaxNPerSource[s2] = maxn[s2];
    for(size_t c = 0; c < cells; ++c) {
        const int32_t keep = std::min(narr[c], mx);
        if(keep < narr[c]) {
            char m[160];
            snprintf(m, sizeof m, "%d arrivals in file at receiver cell %zu, but only memory for %d", narr[c], c, keep);
            say(in, m);
        }
        I.NArr[c] = keep;
        for(int32_t a = 0; a < keep; ++a) I.Arr[c * (size_t)mx + a] = recs[c][a];
    }
}

// ReadOutRay (src/mode/ray.cpp:203-370): header (title, frequency, source
// and angle counts, boundary depths, 'rz' or 'xyz'), then per ray its
// take-off angle, its point count with the last point's bounce counts, and
// its points. Nx2D rays (xyz in the file) come back in their plane's
// (range from the first point, depth) coordinates.
template<bool O3D, bool R3D> void read_rays(Internal &in, bhcParams<O3D> &params, bhcOutputs<O3D, R3D> &outputs,
                                            const std::string &path)
{
    ListIn L(path);
    L.list();
    set_title(params.Title, L.token().c_str());
    L.list();
    params.freqinfo->freq0 = L.real();
    L.list();
    const int32_t nsx = L.integer(), nsy = L.integer(), nsz = L.integer();
    if(nsx != params.Pos->NSx || nsy != params.Pos->NSy || nsz != params.Pos->NSz) {
        char m[160];
        snprintf(m, sizeof m, "NSx = %d, NSy = %d, NSz = %d in the ray file, but %d, %d, %d in the setup", nsx, nsy,
                 nsz, params.Pos->NSx, params.Pos->NSy, params.Pos->NSz);
        say(in, m);
    }
    L.list();
    (void)L.integer();
    (void)L.integer();
    L.list();
    (void)L.real();
    (void)L.real();
    L.list();
    const std::string dim = L.token();
    if(dim != (O3D ? "xyz" : "rz"))
        throw std::runtime_error("dimensionality in the ray file is '" + dim + "', must be " + (O3D ? "'xyz'" : "'rz'"));
    struct One {
        double alpha;
        int32_t n, ntop, nbot;
        std::vector<double> pts;
    };
    std::vector<One> rays;
    const int nc = O3D ? 3 : 2;
    while(!L.eof()) {
        One r;
        L.list();
        r.alpha = L.real();
        if(!std::isfinite(r.alpha)) break;
        L.list();
        r.n = L.integer();
        r.ntop = L.integer();
        r.nbot = L.integer();
        if(r.n <= 0) throw std::runtime_error("<= 0 points in a ray of the ray file");
        if(r.ntop < 0 || r.nbot < 0) throw std::runtime_error("invalid number of bounces in a ray of the ray file");
        r.pts.resize((size_t)r.n * nc);
        for(int32_t k = 0; k < r.n; ++k) {
            L.list();
            for(int c = 0; c < nc; ++c) r.pts[(size_t)k * nc + c] = L.real();
        }
        rays.push_back(std::move(r));
    }
    free_outputs(outputs);
    outputs.arrinfo = new ArrInfo{};
    outputs.eigen = new EigenInfo{};
    outputs.rayinfo = new RayInfo<O3D, R3D>{};
    RayInfo<O3D, R3D> &RI = *outputs.rayinfo;
    RI.NRays = (int32_t)rays.size();
    RI.results = new RayResult<O3D, R3D>[rays.size() ? rays.size() : 1]();
    for(size_t i = 0; i < rays.size(); ++i) {
        const One &r = rays[i];
        RayResult<O3D, R3D> &res = RI.results[i];
        res.Nsteps = r.n;
        res.SrcDeclAngle = O3D ? r.alpha * (180.0 / kPi) : r.alpha;
        res.ray = new rayPt<R3D>[r.n]();
        double tx = 1.0, ty = 0.0;
        if constexpr(O3D && !R3D) {
            // the plane's radial direction: first to last point (OceanToRayX)
            const double *p0 = &r.pts[0], *p1 = &r.pts[(size_t)(r.n - 1) * 3];
            const double dx = p1[0] - p0[0], dy = p1[1] - p0[1], l = std::sqrt(dx * dx + dy * dy);
            if(l > 0) { tx = dx / l; ty = dy / l; }
        }
        for(int32_t k = 0; k < r.n; ++k) {
            const double *q = &r.pts[(size_t)k * nc];
            if constexpr(!O3D) {
                res.ray[k].x.x = q[0];
                res.ray[k].x.y = q[1];
            } else if constexpr(R3D) {
                res.ray[k].x.x = q[0];
                res.ray[k].x.y = q[1];
                res.ray[k].x.z = q[2];
            } else {
                res.ray[k].x.x = (q[0] - r.pts[0]) * tx + (q[1] - r.pts[1]) * ty;
                res.ray[k].x.y = q[2];
            }
        }
        res.ray[r.n - 1].NumTopBnc = r.ntop;
        res.ray[r.n - 1].NumBotBnc = r.nbot;
    }
}

template<typename F> auto guard(const char *what, const void *internal, F &&fn) -> decltype(fn())
{
    try {
        return fn();
    } catch(const std::exception &e) {
        const std::string m = std::string("bhc::") + what + ": " + e.what();
        if(internal) {
            say(*state(internal), m);
            state(internal)->error = m;
        } else {
            std::printf("%s\n", m.c_str());
        }
        return decltype(fn())(false);
    }
}

} // namespace

// ------------------------------------------------------------------ setup
// the parameters' summary that setup and echo write as PRT text
template<bool O3D> std::string echo_text(const bhcParams<O3D> &params)
{
    std::ostringstream o;
    o << "bhcb (B200) - " << params.Title << "\n";
    o << " frequency = " << params.freqinfo->freq0 << " Hz\n";
    o << " number of sources = " << params.Pos->NSz << ", receiver depths = " << params.Pos->NRz
      << ", receiver ranges = " << params.Pos->NRr << "\n";
    if(!O3D) {
        o << " SSP type '" << params.ssp->Type << "', " << params.ssp->NPts << " points, depth "
          << params.Bdry->Bot.hs.Depth << " m\n";
        o << " run type '" << std::string(params.Beam->RunType, 7) << "', beams " << params.Angles->alpha.n
          << "\n";
    }
    return o.str();
}

template<bool O3D, bool R3D> bool setup(const bhcInit &init, bhcParams<O3D> &params, bhcOutputs<O3D, R3D> &outputs)
{
    std::memset(static_cast<void *>(&params), 0, sizeof params);
    std::memset(static_cast<void *>(&outputs), 0, sizeof outputs);
    auto *in = new Internal();
    in->init = init;
    in->root = init.FileRoot ? init.FileRoot : "";
    in->dim = !O3D ? 2 : (R3D ? 3 : 4);
    params.internal = in;
    alloc_params(params);
    if(!init.prtCallback && !in->root.empty()) {
        in->prt.open(in->root + ".prt");
        if(!in->prt.is_open()) say(*in, "could not open print file " + in->root + ".prt");
    }
    return guard("setup", in, [&]() -> bool {
        if constexpr(!O3D) {
            if(!in->root.empty()) {
                char msg[512];
                bhcb_env_desc *d = nullptr;
                if(bhcb_read_env_desc(in->root.c_str(), &d, msg, sizeof msg) != BHCB_OK)
                    throw std::runtime_error(msg);
                params_from_desc(params, *d);
                bhcb_free_env_desc(d);
            } else {
                std::vector<double> z, c, one, zero, rr, al;
                std::vector<float> sz, rz;
                bhcb_env_desc d;
                default_desc_2d(z, c, one, zero, sz, rz, rr, al, d);
                params_from_desc(params, d);
            }
        } else {
            // 3-D / Nx2D: the setup's values for inspection (run reads the files)
            if(in->root.empty()) throw std::runtime_error("3-D and Nx2D setups need FileRoot");
            int32_t dims[6] = {0};
            int64_t nrays = 0;
            char msg[512];
            if(bhcb_check_env3d(in->root.c_str(), dims, &nrays, msg, sizeof msg) != BHCB_OK)
                throw std::runtime_error(msg);
            Position &P = *params.Pos;
            P.NSz = dims[0]; P.NSx = dims[1]; P.NSy = dims[2]; P.Ntheta = dims[3]; P.NRz = dims[4]; P.NRr = dims[5];
            P.NRz_per_range = dims[4];
            std::memcpy(params.Beam->RunType, R3D ? "C    3 " : "C    2 ", 7);
            std::ifstream f(in->root + ".env");
            std::string title;
            std::getline(f, title);
            const size_t a = title.find('\''), b = title.rfind('\'');
            set_title(params.Title, (a != std::string::npos && b > a) ? title.substr(a + 1, b - a - 1).c_str() : "");
            double f0 = 0;
            f >> f0;
            params.freqinfo->freq0 = f0;
            // run type letter (first character of the line that ends the run type) for outputs
            std::string line;
            while(std::getline(f, line)) {
                const size_t q = line.find('\'');
                if(q != std::string::npos && line.size() > q + 6 && (line[q + 6] == '3' || line[q + 6] == '2')) {
                    params.Beam->RunType[0] = line[q + 1];
                }
            }
        }
        // the input echo as PRT text (the reference's readers write it while
        // they read); a setup from the defaults without a callback prints none
        if(init.prtCallback || in->prt.is_open()) prt(*in, echo_text(params));
        return true;
    });
}

template<bool O3D> bool echo(bhcParams<O3D> &params)
{
    return guard("echo", params.internal, [&]() -> bool {
        prt(internal_of(params), echo_text(params));
        return true;
    });
}

template<bool O3D, bool R3D> bool run(bhcParams<O3D> &params, bhcOutputs<O3D, R3D> &outputs)
{
    return guard("run", params.internal, [&]() -> bool {
        Internal &in = internal_of(params);
        if(in.worker.joinable()) in.worker.join();
        if(in.blocking) {
            run_now(params, outputs);
            if(in.init.completedCallback) in.init.completedCallback();
            return true;
        }
        // non-blocking (extsetup_blocking(false)): the run continues on a worker
        // thread; postprocess waits for it
        in.ok = true;
        in.progress = 0;
        in.worker = std::thread([&in, &params, &outputs]() {
            try {
                run_now(params, outputs);
            } catch(const std::exception &e) {
                in.ok = false;
                in.error = e.what();
            }
            if(in.init.completedCallback) in.init.completedCallback();
        });
        return true;
    });
}

template<bool O3D, bool R3D> bool postprocess(bhcParams<O3D> &params, bhcOutputs<O3D, R3D> &)
{
    return guard("postprocess", params.internal, [&]() -> bool {
        Internal &in = internal_of(params);
        if(in.worker.joinable()) in.worker.join();
        if(!in.ok) throw std::runtime_error(in.error);
        return true;
    });
}

template<bool O3D> int get_percent_progress(bhcParams<O3D> &params)
{
    if(!params.internal) return 0;
    return state(params.internal)->progress.load();
}

template<bool O3D, bool R3D> bool writeout(const bhcParams<O3D> &params, const bhcOutputs<O3D, R3D> &,
                                           const char *FileRoot)
{
    return guard("writeout", params.internal, [&]() -> bool {
        Internal &in = internal_of(params);
        if(!in.ctx) throw std::runtime_error("writeout before run");
        const std::string root = FileRoot ? FileRoot : in.root;
        if(root.empty()) throw std::runtime_error("no FileRoot to write to");
        check(in.ctx, bhcb_writeout(in.ctx, 0, 0, root.c_str()), "writeout");
        return true;
    });
}

template<bool O3D, bool R3D> bool readout(bhcParams<O3D> &params, bhcOutputs<O3D, R3D> &outputs, const char *FileRoot)
{
    return guard("readout", params.internal, [&]() -> bool {
        if(!FileRoot) throw std::runtime_error("FileRoot is null");
        // the mode of the setup's RunType picks the file (GetMode, src/api.cpp:367-382)
        const char run0 = params.Beam->RunType[0];
        Internal &in = internal_of(params);
        if(run0 == 'A' || run0 == 'a') {
            read_arrivals(in, params, outputs, std::string(FileRoot) + ".arr", run0 == 'A');
            return true;
        }
        if(run0 == 'V' || run0 == 'v') throw std::runtime_error("ReadOutArrivals called while not in arrivals mode");
        if(run0 == 'R') {
            read_rays(in, params, outputs, std::string(FileRoot) + ".ray");
            return true;
        }
        if(run0 == 'E') return true;   // the eigenray mode reads nothing back
        if(run0 != 'C' && run0 != 'S' && run0 != 'I')
            throw std::runtime_error(std::string("invalid RunType ") + run0);
        // .shd (src/mode/tl.cpp:38-248): 10 header records, then one record
        // per (Sx, Sy, bearing, Sz, receiver depth) row of NRr complex values
        ShdReader r(std::string(FileRoot) + ".shd");
        auto h0 = r.rec(0);
        set_title(params.Title, std::string(h0.data() + 4, 80).c_str());
        auto h2 = r.rec(2);
        int32_t v[7];
        std::memcpy(v, h2.data(), 28);
        const int32_t Ntheta = v[1], NSx = v[2], NSy = v[3], NSz = v[4], NRz = v[5], NRr = v[6];
        if(Ntheta < 1 || NSx < 1 || NSy < 1 || NSz < 1 || NRz < 1 || NRr < 1 || (size_t)NRr * 8 > r.lrecl)
            throw std::runtime_error("bad .shd header");
        double f0 = 0;
        std::memcpy(&f0, h2.data() + 28, 8);
        params.freqinfo->freq0 = f0;
        auto sz = r.rec(7), rz = r.rec(8), rr = r.rec(9);
        Position &P = *params.Pos;
        P.NSx = NSx; P.NSy = NSy; P.NSz = NSz; P.NRz = NRz; P.NRr = NRr; P.Ntheta = Ntheta;
        P.NRz_per_range = NRz;
        resize(P.Sz, NSz); std::memcpy(P.Sz, sz.data(), std::min(sz.size(), NSz * sizeof(float)));
        resize(P.Rz, NRz); std::memcpy(P.Rz, rz.data(), std::min(rz.size(), NRz * sizeof(float)));
        resize(P.Rr, NRr); std::memcpy(P.Rr, rr.data(), std::min(rr.size(), NRr * sizeof(double)));
        P.RrInKm = false;
        delete[] outputs.uAllSources;
        const size_t rows = (size_t)NSx * NSy * Ntheta * NSz * NRz;
        outputs.uAllSources = new cpxf[rows * NRr];
        // file rows are [isx][isy][itheta][isz][iz]; the field [isz][isx][isy][itheta][iz]
        size_t k = 10;
        for(int isx = 0; isx < NSx; ++isx)
            for(int isy = 0; isy < NSy; ++isy)
                for(int it = 0; it < Ntheta; ++it)
                    for(int isz = 0; isz < NSz; ++isz)
                        for(int iz = 0; iz < NRz; ++iz, ++k) {
                            auto row = r.rec(k);
                            const size_t dst = ((((size_t)isz * NSx + isx) * NSy + isy) * Ntheta + it) * NRz + iz;
                            std::memcpy(&outputs.uAllSources[dst * NRr], row.data(), NRr * sizeof(cpxf));
                        }
        return true;
    });
}

template<bool O3D> bool writeenv(bhcParams<O3D> &params, const char *FileRoot)
{
    return guard("writeenv", params.internal, [&]() -> bool {
        if(!FileRoot) throw std::runtime_error("FileRoot is null");
        if constexpr(O3D) {
            // 3-D and Nx2D parameters are the setup's files (this library runs
            // them from FileRoot): write them again under the new root
            Internal &in = internal_of(params);
            if(in.root.empty()) throw std::runtime_error("3-D and Nx2D setups need FileRoot");
            bool any = false;
            for(const char *ext : {".env", ".ssp", ".bty", ".ati", ".sbp", ".trc", ".brc"}) {
                std::ifstream src(in.root + ext, std::ios::binary);
                if(!src.good()) continue;
                std::ofstream dst(std::string(FileRoot) + ext, std::ios::binary);
                if(!dst.good()) throw std::runtime_error(std::string("cannot write ") + FileRoot + ext);
                dst << src.rdbuf();
                any = any || std::strcmp(ext, ".env") == 0;
            }
            if(!any) throw std::runtime_error("cannot read " + in.root + ".env");
        } else {
            DescOf d(params);
            write_env_files(d.d, FileRoot);
        }
        return true;
    });
}

template<bool O3D, bool R3D> void finalize(bhcParams<O3D> &params, bhcOutputs<O3D, R3D> &outputs)
{
    if(params.internal) {
        Internal *in = state(params.internal);
        if(in->worker.joinable()) in->worker.join();
        if(in->ctx) bhcb_close(in->ctx);
        delete in;
        params.internal = nullptr;
    }
    free_outputs(outputs);
    free_params(params);
}

template<bool O3D, bool R3D> bool get_ssp(bhcParams<O3D> &params, const VEC23<R3D> &x, float &sound_speed)
{
    return guard("get_ssp", params.internal, [&]() -> bool {
        Internal &in = internal_of(params);
        if constexpr(O3D) {
            // the setup's files' tables, interpolated on the host; an Nx2D
            // point (range, depth) is taken on the plane along x through the
            // origin, (r, 0, z) (the reference's Origin is left unset there)
            if(in.root.empty()) throw std::runtime_error("3-D and Nx2D setups need FileRoot");
            const bhcb::Env3Tables T = bhcb::preprocess3d(bhcb::read_env_files(in.root, true), params.freqinfo->freq0);
            double c;
            if constexpr(R3D) c = bhcb::ssp_at3(T, x.x, x.y, x.z);
            else c = bhcb::ssp_at3(T, x.x, 0.0, x.y);
            sound_speed = (float)c;
        } else {
            // host interpolation of the tables the tracer uses; no GPU needed
            (void)in;
            DescOf d(params);
            const double c = bhcb::ssp_at(bhcb::preprocess(bhcb::env_from_desc(d.d), d.d.freq0), x.x, x.y);
            sound_speed = (float)c;
        }
        return true;
    });
}

// --------------------------------------------------------------- extsetup
template<bool O3D> void extsetup_sxsy(bhcParams<O3D> &p, int32_t NSx, int32_t NSy)
{
    p.Pos->NSx = NSx; p.Pos->NSy = NSy;
    resize(p.Pos->Sx, NSx); resize(p.Pos->Sy, NSy);
}
template<bool O3D> void extsetup_sz(bhcParams<O3D> &p, int32_t NSz)
{
    p.Pos->NSz = NSz;
    resize(p.Pos->Sz, NSz);
}
template<bool O3D> void extsetup_rcvrranges(bhcParams<O3D> &p, int32_t NRr)
{
    p.Pos->NRr = NRr;
    resize(p.Pos->Rr, NRr);
}
template<bool O3D> void extsetup_rcvrdepths(bhcParams<O3D> &p, int32_t NRz)
{
    p.Pos->NRz = NRz;
    if(p.Beam->RunType[4] != 'I') p.Pos->NRz_per_range = NRz;
    resize(p.Pos->Rz, NRz);
}
template<bool O3D> void extsetup_rcvrbearings(bhcParams<O3D> &p, int32_t Ntheta)
{
    p.Pos->Ntheta = Ntheta;
    resize(p.Pos->theta, Ntheta);
}
template<bool O3D> void extsetup_rayelevations(bhcParams<O3D> &p, int32_t n)
{
    p.Angles->alpha.n = n;
    resize(p.Angles->alpha.angles, std::max(n, 2));
}
template<bool O3D> void extsetup_raybearings(bhcParams<O3D> &p, int32_t n)
{
    p.Angles->beta.n = n;
    resize(p.Angles->beta.angles, std::max(n, 2));
}
template<bool O3D> void extsetup_sbp(bhcParams<O3D> &p, int32_t NSBPPts)
{
    p.sbp->NSBPPts = NSBPPts;
    p.sbp->SBPFlag = '*';
    resize(p.sbp->SrcBmPat, 2 * (size_t)NSBPPts);
}
template<bool O3D> void extsetup_freqvec(bhcParams<O3D> &p, int32_t Nfreq)
{
    p.freqinfo->Nfreq = Nfreq;
    resize(p.freqinfo->freqVec, Nfreq);
}
template<bool O3D> void extsetup_altimetry(bhcParams<O3D> &p, const IORI2<O3D> &NPts)
{
    if constexpr(O3D) {
        p.bdinfo->top.NPts = NPts;
        resize(p.bdinfo->top.bd, (size_t)NPts.x * NPts.y);
    } else {
        p.bdinfo->top.NPts = NPts;
        resize(p.bdinfo->top.bd, NPts);
    }
    p.bdinfo->top.dirty = true;
}
template<bool O3D> void extsetup_bathymetry(bhcParams<O3D> &p, const IORI2<O3D> &NPts, const int32_t &NBotProvinces)
{
    if constexpr(O3D) {
        p.bdinfo->bot.NPts = NPts;
        resize(p.bdinfo->bot.bd, (size_t)NPts.x * NPts.y);
    } else {
        p.bdinfo->bot.NPts = NPts;
        resize(p.bdinfo->bot.bd, NPts);
    }
    p.bdinfo->bot.NBotProvinces = NBotProvinces;
    resize(p.bdinfo->bot.BotProv, NBotProvinces);
    p.bdinfo->bot.dirty = true;
}
template<bool O3D> void extsetup_trc(bhcParams<O3D> &p, int32_t NPts)
{
    p.refl->top.NPts = NPts;
    resize(p.refl->top.r, NPts);
}
template<bool O3D> void extsetup_brc(bhcParams<O3D> &p, int32_t NPts)
{
    p.refl->bot.NPts = NPts;
    resize(p.refl->bot.r, NPts);
}
void extsetup_ssp_quad(bhcParams<false> &p, int32_t NPts, int32_t Nr)
{
    p.ssp->NPts = NPts;
    p.ssp->Nz = NPts;
    p.ssp->Nr = Nr;
    p.ssp->Type = 'Q';
    resize(p.ssp->Seg.r, Nr);
    resize(p.ssp->cMat, (size_t)NPts * Nr);
    p.ssp->dirty = true;
}
void extsetup_ssp_hexahedral(bhcParams<true> &p, int32_t Nx, int32_t Ny, int32_t Nz)
{
    p.ssp->Nx = Nx; p.ssp->Ny = Ny; p.ssp->Nz = Nz;
    p.ssp->Type = 'H';
    resize(p.ssp->Seg.x, Nx); resize(p.ssp->Seg.y, Ny); resize(p.ssp->Seg.z, Nz);
    resize(p.ssp->cMat, (size_t)Nx * Ny * Nz);
    resize(p.ssp->czMat, (size_t)Nx * Ny * Nz);
    p.ssp->dirty = true;
}
template<bool O3D> void extsetup_blocking(bhcParams<O3D> &p, const bool &blocking)
{
    if(p.internal) state(p.internal)->blocking = blocking;
}

// ------------------------------------------------------- instantiations
#define BHCB_INST_RUN(O, R)                                                                                  \
    template bool setup<O, R>(const bhcInit &, bhcParams<O> &, bhcOutputs<O, R> &);                        \
    template bool run<O, R>(bhcParams<O> &, bhcOutputs<O, R> &);                                            \
    template bool postprocess<O, R>(bhcParams<O> &, bhcOutputs<O, R> &);                                    \
    template bool writeout<O, R>(const bhcParams<O> &, const bhcOutputs<O, R> &, const char *);             \
    template bool readout<O, R>(bhcParams<O> &, bhcOutputs<O, R> &, const char *);                          \
    template void finalize<O, R>(bhcParams<O> &, bhcOutputs<O, R> &);                                       \
    template bool get_ssp<O, R>(bhcParams<O> &, const VEC23<R> &, float &);
BHCB_INST_RUN(false, false)
BHCB_INST_RUN(true, false)
BHCB_INST_RUN(true, true)
#undef BHCB_INST_RUN
#define BHCB_INST_P(O)                                                                                       \
    template void extsetup_sxsy<O>(bhcParams<O> &, int32_t, int32_t);                                      \
    template void extsetup_sz<O>(bhcParams<O> &, int32_t);                                                  \
    template void extsetup_rcvrranges<O>(bhcParams<O> &, int32_t);                                          \
    template void extsetup_rcvrdepths<O>(bhcParams<O> &, int32_t);                                          \
    template void extsetup_rcvrbearings<O>(bhcParams<O> &, int32_t);                                        \
    template void extsetup_rayelevations<O>(bhcParams<O> &, int32_t);                                       \
    template void extsetup_raybearings<O>(bhcParams<O> &, int32_t);                                         \
    template void extsetup_sbp<O>(bhcParams<O> &, int32_t);                                                 \
    template void extsetup_freqvec<O>(bhcParams<O> &, int32_t);                                             \
    template void extsetup_altimetry<O>(bhcParams<O> &, const IORI2<O> &);                                  \
    template void extsetup_bathymetry<O>(bhcParams<O> &, const IORI2<O> &, const int32_t &);                \
    template void extsetup_trc<O>(bhcParams<O> &, int32_t);                                                 \
    template void extsetup_brc<O>(bhcParams<O> &, int32_t);                                                 \
    template void extsetup_blocking<O>(bhcParams<O> &, const bool &);                                       \
    template bool echo<O>(bhcParams<O> &);                                                                  \
    template int get_percent_progress<O>(bhcParams<O> &);                                                   \
    template bool writeenv<O>(bhcParams<O> &, const char *);
BHCB_INST_P(false)
BHCB_INST_P(true)
#undef BHCB_INST_P

} // namespace bhc
