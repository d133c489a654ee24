// Nx2D field mode (BELLHOP3D's N x 2-D: O3D ocean, 2-D rays), TL runs, FP64.
//
// Each ray lives in the vertical plane of its bearing beta through its source:
// ray coordinates (r, z) map to ocean coordinates by x = xs + r (cos beta,
// sin beta), depth unchanged (RayToOceanX / RayToOceanT / OceanToRayX /
// OceanToRayT, src/common_run.hpp:221-317). The step is the 2-D one (scalar
// p-q) with the sound speed evaluated in the 3-D ocean and projected on the
// plane (src/ssp.hpp:446-463), the step-size reduction and boundary landing
// solved in ocean coordinates against the 3-D boundary grids
// (src/step.hpp:654-811, O3D branch), and reflection off the 3-D triangle
// normal projected on the plane with the 3-D halfspace coefficient
// (src/reflect.hpp:125-452). The influence is the 2-D Cartesian geometric one
// (src/influence.hpp:1201-1406) on the ray's own receiver bearing: beams are
// launched along the receiver bearings (src/module/rayangles.hpp:163-179).
//
//  trace_nx_kernel      one ray per thread: RayInit / RayUpdate / RayTerminate
//                       of the Nx2D path and the sequential part of the 2-D
//                       influence; one record per segment that brackets
//                       receiver ranges.
//  influence_nx_kernel  one thread per (record, receiver depth); contributions
//                       added into the [isz][isx][isy][itheta][iz][ir] field.
//  scale_nx_kernel      ScalePressure, 2-D form (src/influence.hpp:1556-1627).
//
// This file is compiled without multiply-add contraction (-fmad=false) and
// takes the plane's (cos beta, sin beta) and the launch (cos alpha, sin alpha)
// from host tables: the landing on an x or y grid line of the boundary
// (OceanToRayX's ulp nudges towards the forward side, at most four) decides
// whether the next step starts in the new cell or first takes a forced small
// step, and that decision follows the last bits of the ocean position. With
// separately rounded products and sums and the same direction doubles, those
// bits follow the reference's own arithmetic.
#include <cuda_runtime.h>

#include "bhcb_internal.h"
#include "device_math.cuh"
#include "trace2d.cuh"
#include "influence2d.cuh"
#include "ray2d.cuh"
#include "trace3d.cuh"

namespace bhcb {

namespace {

typedef RayPt<double> RayN;

struct OrgN {   // Origin<true, false>: source position and the radial direction
    V3 xs;
    double tx, ty;
};

__device__ __forceinline__ V3 to_ocean_x(V2<double> x, const OrgN &o)
{
    return v3(o.xs.x + x.x * o.tx, o.xs.y + x.x * o.ty, x.y);
}
__device__ __forceinline__ V3 to_ocean_t(V2<double> t, const OrgN &o) { return v3(t.x * o.tx, t.x * o.ty, t.y); }
__device__ __forceinline__ V2<double> to_ray_t(V3 t, const OrgN &o) { return mk2(t.x * o.tx + t.y * o.ty, t.z); }

// the floating-point value k representations away (RealBitsAddInt)
__device__ __forceinline__ double bits_add(double v, long long k)
{
    return __longlong_as_double(__double_as_longlong(v) + k);
}

// OceanToRayX (src/common_run.hpp:244-302): range from the larger radial
// component; when the landing coordinate snap was x or y, nudge the range by
// ulps (at most 4) until the point maps back on the forward side of it
__device__ V2<double> to_ray_x(V3 x, const OrgN &o, V2<double> t, int snap, RunCounters *ctr)
{
    V2<double> r;
    r.y = x.z;
    r.x = fabs(o.tx) >= fabs(o.ty) ? (x.x - o.xs.x) / o.tx : (x.y - o.xs.y) / o.ty;
    if(snap < -2 || snap == -1 || snap >= 2) return r;
    for(int i = 0; i < 4; ++i) {
        const V3 xb = to_ocean_x(r, o);
        const double wx = o.tx * t.x, wy = o.ty * t.x;
        const double ex = xb.x - x.x, ey = xb.y - x.y;
        const bool okx = wx * ex >= 0.0, oky = wy * ey >= 0.0;
        if((snap == 0 && okx) || (snap == 1 && oky) || (okx && oky)) return r;
        r.x = bits_add(r.x, t.x > 0.0 ? 1 : -1);
    }
    run_warn(ctr, WARN_OCEANTORAYX_GAVEUP);
    return r;
}

// EvaluateSSP<O3D = true, R3D = false> (src/ssp.hpp:376-463): the 3-D sound
// speed at the ocean point, its gradient and curvature projected on the plane
template<bool NEED_RHO = false> __device__ __forceinline__ void eval_ssp_nx(V2<double> x, V2<double> t,
                                                                           SSPOut<double> &o, const Env3Dev &E,
                                                                           const OrgN &org, Seg3 &s,
                                                                           RunCounters *ctr)
{
    SSPOut3 p;
    eval_ssp3<NEED_RHO>(to_ocean_x(x, org), to_ocean_t(t, org), p, E, s, ctr);
    o.gradc = mk2(org.tx * p.gradc.x + org.ty * p.gradc.y, p.gradc.z);
    o.crz = org.tx * p.cxz + org.ty * p.cyz;
    o.crr = p.cxx * org.tx * org.tx + FLTD(2.0) * p.cxy * org.tx * org.ty + p.cyy * org.ty * org.ty;
    o.c = p.c;
    o.ci = p.ci;
    o.rho = p.rho;
    o.czz = p.czz;
}

// Step, Nx2D (src/step.hpp:654-811 with R3D = false, O3D = true)
__device__ void step_nx(const RayN &ray0, RayN &ray2, Bd3 &top, Bd3 &bot, const OrgN &org, const Env3Dev &E,
                        Seg3 &iSeg, int &small, bool &tr, bool &br, RunCounters *ctr)
{
    SSPOut<double> o0, o1, o2;
    eval_ssp_nx(ray0.x, ray0.t, o0, E, org, iSeg, ctr);
    const double cnn0 = o0.crr * ray0.t.y * ray0.t.y - 2.0 * o0.crz * ray0.t.x * ray0.t.y
        + o0.czz * ray0.t.x * ray0.t.x;
    const V2<double> pq0p = scl2(-cnn0, ray0.q), pq0q = scl2(o0.c, ray0.p);
    const Seg3 s0 = iSeg;
    const double csq0 = o0.c * o0.c;
    const V2<double> u0 = scl2(o0.c, ray0.t);
    double h = E.deltas;
    const V3 x_o = to_ocean_x(ray0.x, org);
    reduce_step3(x_o, to_ocean_t(u0, org), s0, top, bot, org.xs, E, h, small, ctr);
    const double halfh = 0.5 * h;
    RayN ray1;
    ray1.x = add2(ray0.x, scl2(halfh, u0));
    ray1.t = sub2(ray0.t, div2(scl2(halfh, o0.gradc), csq0));
    ray1.p = add2(ray0.p, scl2(halfh, pq0p));
    ray1.q = add2(ray0.q, scl2(halfh, pq0q));

    eval_ssp_nx(ray1.x, ray1.t, o1, E, org, iSeg, ctr);
    const double cnn1 = o1.crr * ray1.t.y * ray1.t.y - 2.0 * o1.crz * ray1.t.x * ray1.t.y
        + o1.czz * ray1.t.x * ray1.t.x;
    const V2<double> pq1p = scl2(-cnn1, ray1.q), pq1q = scl2(o1.c, ray1.p);
    const double csq1 = o1.c * o1.c;
    const V2<double> u1 = scl2(o1.c, ray1.t);
    reduce_step3(x_o, to_ocean_t(u1, org), s0, top, bot, org.xs, E, h, small, ctr);
    const double w1 = h / (2.0 * halfh);
    const double w0 = 1.0 - w1;
    const V2<double> u2 = add2(scl2(w0, u0), scl2(w1, u1));
    V3 x2_o;
    int snap;
    step_to_bdry3(x_o, x2_o, to_ocean_t(u2, org), h, tr, br, s0, top, bot, org.xs, E, ctr, snap);
    ray2.x = to_ray_x(x2_o, org, u2, snap, ctr);
    const double hw0 = h * w0, hw1 = h * w1;
    ray2.t = sub2(sub2(ray0.t, div2(scl2(hw0, o0.gradc), csq0)), div2(scl2(hw1, o1.gradc), csq1));
    const Cx<double> d0 = o0.ci == 0.0 ? cx<double>(hw0 / o0.c, 0.0) : rdivc(hw0, cx<double>(o0.c, o0.ci));
    const Cx<double> d1 = o1.ci == 0.0 ? cx<double>(hw1 / o1.c, 0.0) : rdivc(hw1, cx<double>(o1.c, o1.ci));
    ray2.taur = ray0.taur + d0.r + d1.r;
    ray2.taui = ray0.taui + d0.i + d1.i;
    ray2.p = add2(add2(ray0.p, scl2(hw0, pq0p)), scl2(hw1, pq1p));
    ray2.q = add2(add2(ray0.q, scl2(hw0, pq0q)), scl2(hw1, pq1q));
    ray2.Amp = ray0.Amp;
    ray2.Phase = ray0.Phase;
    ray2.ntop = ray0.ntop;
    ray2.nbot = ray0.nbot;
    eval_ssp_nx(ray2.x, ray2.t, o2, E, org, iSeg, ctr);
    ray2.c = o2.c;
    if(iSeg.z != s0.z) {   // CurvatureCorrection, 2-D form, depth crossings only
        const V2<double> gj = sub2(o2.gradc, o0.gradc);
        const V2<double> n2 = mk2(-ray2.t.y, ray2.t.x);
        const double cnj = dot2(gj, n2), csj = dot2(gj, ray2.t);
        const double rm = ray2.t.x / ray2.t.y;
        const double rn = rm * (2.0 * cnj - rm * csj) / ray2.c;
        ray2.p = sub2(ray2.p, scl2(rn, ray2.q));
    }
}

// Reflect, Nx2D (src/reflect.hpp:125-452, O3D && !R3D): the 3-D boundary
// normal projected on the plane; kappa the boundary curvature along the plane
// (OceanToRayCurvature, src/reflect.hpp:94-121; 0 for flat triangles)
__device__ void reflect_nx(const RayN &old, RayN &np, const HsDev &hs, bool istop, V3 nB3, double kappa,
                           const Env3Dev &E, const OrgN &org, Seg3 &iSeg, RunCounters *ctr)
{
    V2<double> nB = to_ray_t(nB3, org);
    nB = scl2(1.0 / sqrt(dot2(nB, nB)), nB);
    const double Th = dot2(old.t, nB);
    V2<double> tB = sub2(old.t, scl2(Th, nB));
    tB = scl2(1.0 / sqrt(dot2(tB, tB)), tB);
    const double Tg = dot2(old.t, tB);
    np.ntop = old.ntop + (istop ? 1 : 0);
    np.nbot = old.nbot + (istop ? 0 : 1);
    np.x = old.x;
    np.t = sub2(old.t, scl2(2.0 * Th, nB));
    SSPOut<double> o;
    eval_ssp_nx<true>(old.x, np.t, o, E, org, iSeg, ctr);
    const double c = o.c;
    np.c = c;
    np.taur = old.taur;
    np.taui = old.taui;
    const V2<double> rayt = scl2(c, old.t), rayn = mk2(-rayt.y, rayt.x);
    const V2<double> rayt_t = scl2(c, np.t), rayn_t = mk2(rayt_t.y, -rayt_t.x);
    double rn = FLTD(2.0) * kappa / (c * c) / Th;
    double cnjump = -dot2(o.gradc, sub2(rayn_t, rayn));
    const double csjump = -dot2(o.gradc, sub2(rayt_t, rayt));
    if(istop) { cnjump = -cnjump; rn = -rn; }
    const double rm = Tg / Th;
    rn += rm * (2.0 * cnjump - rm * csjump) / (c * c);
    if(E.e1d.beam2 == 'D') rn *= 2.0;
    else if(E.e1d.beam2 == 'Z') rn = 0.0;
    np.p = add2(old.p, scl2(rn, old.q));
    np.q = old.q;
    if(hs.bc == 'R') {
        np.Amp = old.Amp;
        np.Phase = old.Phase;
    } else if(hs.bc == 'V') {
        np.Amp = old.Amp;
        np.Phase = old.Phase + BHCB_PI;
    } else if(hs.bc == 'F') {
        double theta = (180.0 / BHCB_PI) * fabs(atan2(Th, Tg));
        if(theta > 90.0) theta = 180.0 - theta;
        double rc, ph;
        refl_coef(istop ? E.e1d.trc : E.e1d.brc, istop ? E.e1d.ntrc : E.e1d.nbrc, theta, rc, ph, ctr);
        np.Amp = old.Amp * rc;
        np.Phase = old.Phase + ph;
    } else if(hs.bc == 'A' || hs.bc == 'G') {   // halfspace, gamma form of the 3-D ocean
        const double omega = FLTD(2.0) * BHCB_PI * E.freq0;
        const double gk = omega * Tg;
        const double wc = omega / c;
        const Cx<double> g1sq = cx<double>(wc * wc - gk * gk, -DBL_MIN_POS);
        const Cx<double> wP = rdivc(omega, cx<double>(hs.cPr, hs.cPi));
        Cx<double> g2sq = csub(cmul(wP, wP), cx<double>(gk * gk, 0.0));
        g2sq.i -= DBL_MIN_POS;
        const Cx<double> g1 = csqrt_(cx<double>(-g1sq.r, -g1sq.i));
        const Cx<double> g2 = csqrt_(cx<double>(-g2sq.r, -g2sq.i));
        const Cx<double> a = cscl(hs.rho, g1), b = cscl(o.rho, g2);
        const Cx<double> Refl = cdiv(csub(a, b), cadd(a, b));
        const double ar = cabs_(Refl);
        if(ar < FLTD(1.0e-5)) {
            np.Amp = 0.0;
            np.Phase = old.Phase;
        } else {
            np.Amp = ar * old.Amp;
            np.Phase = old.Phase + atan2(Refl.i, Refl.r);
        }
    } else {
        run_error(ctr, ERR_BOUNDARY_CONDITION_TYPE);
        np.Amp = NAN;
        np.Phase = NAN;
    }
}

struct RayStateN {
    RayN p0;
    Bd3 top, bot;
    Seg3 iSeg;
    OrgN org;
    double alpha, c;
    double minx, miny, maxx, maxy;
};

// RayInit, Nx2D (src/trace.hpp:76-266)
__device__ bool ray_init_nx(const Env3Dev &E, const Job3 &J, RayStateN &st, RunCounters *ctr)
{
    const double alpha = E.alpha[J.ialpha];
    st.alpha = alpha;
    const double SrcDecl = (180.0 / BHCB_PI) * alpha;
    st.iSeg = Seg3{0, 0, 0};
    const V3 xs = v3(E.sx[J.isx], E.sy[J.isy], (double)E.sz[J.isz]);
    SSPOut3 o;
    eval_ssp3(xs, v3(0.0, 0.0, 1.0), o, E, st.iSeg, ctr);
    const double c = o.c;
    st.c = c;
    st.org.xs = xs;
    st.org.tx = E.bcs[2 * J.ibeta];
    st.org.ty = E.bcs[2 * J.ibeta + 1];
    const int ibp = min(bsearch_leq2(E.sbp, E.nsbp, SrcDecl), E.nsbp - 2);
    const double s = (SrcDecl - E.sbp[2 * ibp]) / (E.sbp[2 * (ibp + 1)] - E.sbp[2 * ibp]);
    float amp0 = (float)((FLTD(1.0) - s) * E.sbp[2 * ibp + 1] + s * E.sbp[2 * (ibp + 1) + 1]);
    if(E.run0 == 'S') {
        const float om = (float)(FLTD(2.0) * BHCB_PI * E.freq0);
        amp0 = (float)(amp0 * ((double)sqrtf(2.0f) * fabs(sin(om / c * xs.z * sin(alpha)))));
    }
    RayN &p0 = st.p0;
    p0.x = mk2(0.0, xs.z);
    p0.c = c;
    p0.t = mk2(E.acs[2 * J.ialpha] / c, E.acs[2 * J.ialpha + 1] / c);
    p0.taur = p0.taui = 0.0;
    p0.Amp = (double)amp0;
    p0.Phase = 0.0;
    p0.ntop = p0.nbot = 0;
    p0.p = mk2(1.0, 0.0);
    p0.q = mk2(0.0, 1.0);
    st.top.ix = st.top.iy = st.bot.ix = st.bot.iy = 0;
    st.top.justSteppedTo = st.bot.justSteppedTo = false;
    st.top.side = st.bot.side = false;
    st.top.outgoingSide = st.bot.outgoingSide = false;
    const V3 t_o = to_ocean_t(p0.t, st.org);
    get_bdry_seg3(xs, t_o, st.top, E.btop, E.top_nx, E.top_ny, true, true, ctr);
    get_bdry_seg3(xs, t_o, st.bot, E.bbot, E.bot_nx, E.bot_ny, false, true, ctr);
    double dTop, dBot;
    distances3(xs, st.top, st.bot, dTop, dBot);
    if(dTop <= 0.0 || dBot <= 0.0) {
        run_warn(ctr, WARN_SOURCE_OUTSIDE_BOUNDARIES);
        return false;
    }
    const Bdry3PtDev *bb = E.bbot, *bt = E.btop;
    st.minx = max(bb[0].x[0], bt[0].x[0]);
    st.miny = max(bb[0].x[1], bt[0].x[1]);
    st.maxx = min(bb[(size_t)(E.bot_nx - 1) * E.bot_ny].x[0], bt[(size_t)(E.top_nx - 1) * E.top_ny].x[0]);
    st.maxy = min(bb[E.bot_ny - 1].x[1], bt[E.top_ny - 1].x[1]);
    return true;
}

// RayUpdate, Nx2D (src/trace.hpp:274-381)
__device__ bool ray_update_nx(RayStateN &st, RayN &p1, RayN &p2, int &small, const Env3Dev &E, RunCounters *ctr)
{
    bool tr = false, br = false;
    step_nx(st.p0, p1, st.top, st.bot, st.org, E, st.iSeg, small, tr, br, ctr);
    const V3 x_o = to_ocean_x(p1.x, st.org), t_o = to_ocean_t(p1.t, st.org);
    get_bdry_seg3(x_o, t_o, st.top, E.btop, E.top_nx, E.top_ny, true, false, ctr);
    get_bdry_seg3(x_o, t_o, st.bot, E.bbot, E.bot_nx, E.bot_ny, false, false, ctr);
    const bool two = tr || br;
    if(two) {
        const Bd3 &b = tr ? st.top : st.bot;
        V3 nI = b.n;
        double kappa = 0.0;
        if(tr ? E.top_curv : E.bot_curv) {   // curvilinear grid (src/trace.hpp:318-341)
            const Bdry3PtDev *bd = tr ? E.btop : E.bbot;
            const int ny = tr ? E.top_ny : E.bot_ny;
            const double s1 = (x_o.x - b.x.x) / (b.xmax - b.xmin), s2 = (x_o.y - b.x.y) / (b.ymax - b.ymin);
            const double m1 = 1.0 - s1, m2 = 1.0 - s2;
            const Bdry3PtDev &d00 = bd[(size_t)b.ix * ny + b.iy], &d01 = bd[(size_t)b.ix * ny + b.iy + 1];
            const Bdry3PtDev &d10 = bd[(size_t)(b.ix + 1) * ny + b.iy], &d11 = bd[(size_t)(b.ix + 1) * ny + b.iy + 1];
            nI = v3(d00.noden[0] * m1 * m2 + d10.noden[0] * s1 * m2 + d11.noden[0] * s1 * s2 + d01.noden[0] * m1 * s2,
                    d00.noden[1] * m1 * m2 + d10.noden[1] * s1 * m2 + d11.noden[1] * s1 * s2 + d01.noden[1] * m1 * s2,
                    d00.noden[2] * m1 * m2 + d10.noden[2] * s1 * m2 + d11.noden[2] * s1 * s2 + d01.noden[2] * m1 * s2);
            const double tx = st.org.tx, ty = st.org.ty;
            kappa = d00.kxx * tx * tx + FLTD(2.0) * d00.kxy * tx * ty + d00.kyy * ty * ty;
            if(tr) kappa = -kappa;
        }
        reflect_nx(p1, p2, tr ? E.top : E.bot, tr, nI, kappa, E, st.org, st.iSeg, ctr);
    }
    return two;
}

// RayTerminate, Nx2D (src/trace.hpp:391-477, O3D branch)
__device__ __forceinline__ bool ray_stops_nx(const RayStateN &st, int small, const Env3Dev &E)
{
    const V3 x = to_ocean_x(st.p0.x, st.org), t = to_ocean_t(st.p0.t, st.org);
    const V3 xs = st.org.xs;
    const bool leftbox = fabs(x.x - xs.x) >= E.box_x || fabs(x.y - xs.y) >= E.box_y || fabs(x.z) >= E.box_z;
    const bool esc0 = x.x < st.minx || x.y < st.miny || (x.x == st.minx && t.x < 0.0) || (x.y == st.miny && t.y < 0.0);
    const bool escN = x.x > st.maxx || x.y > st.maxy || (x.x == st.maxx && t.x > 0.0) || (x.y == st.maxy && t.y > 0.0);
    const bool lost = st.p0.Amp < FLTD(0.005);
    return leftbox || lost || esc0 || escN || small > 50;
}

struct CursorN {
    unsigned long long next = 0, end = 0;
};

__device__ __forceinline__ void emit_nx(const SegRec<double> &rec, SegRec<double> *segs, unsigned long long cap,
                                        RunCounters *ctr, CursorN &cur, bool &overflow)
{
    if(cur.next == cur.end) {
        const unsigned long long b = atomicAdd(&ctr->nseg, 32ull);
        if(b + 32 > cap) {
            overflow = true;
            return;
        }
        cur.next = b;
        cur.end = b + 32;
    }
    const uint4 *src = reinterpret_cast<const uint4 *>(&rec);
    uint4 *dst = reinterpret_cast<uint4 *>(segs + cur.next++);
#pragma unroll
    for(int k = 0; k < (int)(sizeof(SegRec<double>) / 16); ++k) dst[k] = src[k];
}

__global__ void __launch_bounds__(64) trace_nx_kernel(const GroupDev *__restrict__ groups, int ngroups,
                                                      long long job_end, SegRec<double> *segs, unsigned long long cap,
                                                      RunCounters *ctr, unsigned long long *job_counter)
{
    for(;;) {
        const long long job = (long long)atomicAdd(job_counter, 1ull);
        if(job >= job_end) break;
        const GroupDev &G = groups[find_group(groups, ngroups, job)];
        const Env3Dev &E = *G.env3;
        const Job3 J = job_indices3(E, (int)(job - G.job_base));
        if(J.isz >= E.nsz) { run_error(ctr, ERR_RAYINIT); continue; }
        RayStateN st;
        if(!ray_init_nx(E, J, st, ctr)) continue;
        RayN &p0 = st.p0;
        RayN p1, p2;
        // Init_Influence, 2-D Cartesian geometric (src/influence.hpp:525-644)
        const EnvDev &e = E.e1d;   // the receiver ranges and beam flags of the plane
        double ratio1 = sqrt(fabs(cos(st.alpha)));
        if(e.gaussian) ratio1 /= sqrt(FLTD(2.0) * BHCB_PI);
        const double rcp_q0 = E.dalpha / st.c;
        InflState inf;
        inf.phase = 0.0;
        inf.qOld = p0.q.x;
        inf.x = p0.x;
        inf.ir = bsearch_gt(e.rr, e.nrr, p0.x.x);
        if(p0.t.x < 0.0 && inf.ir > 0) --inf.ir;
        int small = 0, is = 0;
        bool overflow = false;
        unsigned long long nsteps = 0;
        CursorN cur;
        for(;;) {
            if((nsteps & 31) == 0 && __ldcg(&ctr->err_bits) != 0u) break;
            const bool two = ray_update_nx(st, p1, p2, small, E, ctr);
            ++nsteps;
            SegRec<double> rec;
            if(infl_prologue(p0, p1, inf, e, rcp_q0, ratio1, (int)job, is, rec))
                emit_nx(rec, segs, cap, ctr, cur, overflow);
            ++is;
            if(two) {
                if(infl_prologue(p1, p2, inf, e, rcp_q0, ratio1, (int)job, is, rec))
                    emit_nx(rec, segs, cap, ctr, cur, overflow);
                p0 = p2;
                ++is;
            } else {
                p0 = p1;
            }
            if(overflow) {
                atomicMin(&ctr->overflow_job, (unsigned int)job);
                run_error(ctr, ERR_SEG_OVERFLOW);
                break;
            }
            if(ray_stops_nx(st, small, E)) break;
            if(is >= MAXN_STEPS - 3) {
                run_warn(ctr, WARN_ONERAY_OUTOFMEMORY);
                break;
            }
        }
        for(; cur.next < cur.end; ++cur.next) segs[cur.next].job = -1;
        atomicAdd(&ctr->nsteps, nsteps);
    }
}

// InfluenceGeoCore + ApplyContribution, 2-D Cartesian (src/influence.hpp:
// 423-473, 897-1024), one thread per (record, receiver depth) over the
// record's receiver ranges, within the segment's depth window
// (src/influence.hpp:1285-1292)
__global__ void __launch_bounds__(128) influence_nx_kernel(const SegRec<double> *__restrict__ segs,
                                                           unsigned long long cap,
                                                           const GroupDev *__restrict__ groups, int ngroups,
                                                           float2 *field, RunCounters *ctr, int nzmax)
{
    const unsigned long long nseg = min(__ldcg(&ctr->nseg), cap);
    const unsigned long long nitems = nseg * (unsigned long long)nzmax;
    unsigned int evals = 0;
    for(unsigned long long it = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; it < nitems;
        it += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned long long k = it / (unsigned)nzmax;
        const int iz = (int)(it - k * (unsigned)nzmax);
        const SegRec<double> &S = segs[k];
        if(S.job < 0) continue;
        const GroupDev &G = groups[find_group(groups, ngroups, S.job)];
        const Env3Dev &E = *G.env3;
        if(iz >= E.nrz) continue;
        const bool gauss = E.gaussian != 0, coherent = E.coherent != 0;
        const double freq = E.freq0, omega = FLTD(2.0) * BHCB_PI * freq;
        double sig = S.sigma_seg, fl = 0.0;
        if(gauss) {   // AdjustSigma (src/influence.hpp:91-100)
            fl = min(FLTD(0.2) * freq * S.tau1r, BHCB_PI * (S.c0 / freq));
            sig = max(sig, fl);
        }
        const double zr = (double)E.rz[iz];
        if(fabs(S.tx) > FLTD(0.50001)) {
            const double rmax = (gauss ? 4.0 : 1.0) * sig;
            if(zr < S.zlo - rmax || zr > S.zhi + rmax) continue;
        }
        const Job3 J = job_indices3(E, (int)((long long)S.job - G.job_base));
        float2 *row = field + G.field_base
            + ((((long long)J.isz * E.nsx + J.isx) * E.nsy + J.isy) * E.ntheta + J.ibeta) * E.nrz * E.nrr
            + (long long)iz * E.nrr;
        const double dz = zr - S.x0z;
        for(int ir = S.ir_lo; ir <= S.ir_hi; ++ir) {
            const double dr = E.rr[ir] - S.x0r;
            const double s = (dr * S.tx + dz * S.tz) / S.rlen;
            const double n1 = fabs(dz * S.tx - dr * S.tz);
            const double qF = S.q0 + s * S.dq;
            double sigma = fabs(qF * S.rcp_q0);
            const double sig0 = sigma;
            if(gauss) sigma = max(sigma, fl);
            if(n1 >= (gauss ? 4.0 : 1.0) * sigma) continue;
            const double cnst = S.cnst_num / sqrt(fabs(qF));
            const double w = gauss ? exp(FLTD(-0.5) * (n1 / sigma) * (n1 / sigma)) * (sig0 / sigma)
                                   : (sigma - n1) / sigma;
            const bool caustic = (qF <= 0.0 && S.q0 > 0.0) || (qF >= 0.0 && S.q0 < 0.0);
            const double ph = caustic ? S.phase_b : S.phase_a;
            const double di = S.tau0i + s * S.dtaui;
            float2 v;
            if(coherent) {
                const double amp = cnst * w * exp(omega * di);
                double sn, cs;
                sincos(reduce_2pi(omega * (S.tau0r + s * S.dtaur) - ph), &sn, &cs);
                v = make_float2((float)(amp * cs), (float)(-amp * sn));
            } else {
                double vv = cnst * exp(omega * di);
                vv = vv * vv * w;
                if(gauss) vv *= sqrt(FLTD(2.0) * BHCB_PI);
                v = make_float2((float)vv, 0.f);
            }
            atomicAdd(row + ir, v);
            ++evals;
        }
    }
    for(int o = 16; o > 0; o >>= 1) evals += __shfl_xor_sync(0xffffffffu, evals, o);
    if((threadIdx.x & 31) == 0 && evals) atomicAdd(&ctr->nevals, (unsigned long long)evals);
}

// Arrivals, Nx2D: the contributions of influence_nx_kernel as arrival
// candidates (ApplyContribution with itheta = ibeta and AddArr,
// src/influence.hpp:434-451; ReceiverAngles 2-D form, src/influence.hpp:
// 123-136: receiver azimuth = the source azimuth) keyed (receiver cell, ray,
// step) for the shared radix sort and per-cell replay. With kb.eigen, the same
// contributions as eigen hits (RecordEigenHit with itheta = ibeta), keyed
// (trace group, ray, step, walk position of the receiver range, bearing,
// depth): the 2-D Cartesian walk visits the bracketed ranges towards point1,
// then the depths (src/influence.hpp:1295-1406). One thread per record.
// COUNT: counts into ctr->nevals; otherwise candidate i at atomicAdd(cursor).
template<bool COUNT>
__global__ void __launch_bounds__(128) arr_gather_nx_kernel(const SegRec<double> *__restrict__ segs,
                                                            unsigned long long cap,
                                                            const GroupDev *__restrict__ groups, int ngroups,
                                                            ArrCand *cands, uint64_t *keys, uint32_t *vals,
                                                            unsigned long long cand_cap, unsigned long long *cursor,
                                                            RunCounters *ctr, ArrKeyBits kb)
{
    const unsigned long long nseg = min(__ldcg(&ctr->nseg), cap);
    unsigned long long count = 0;
    for(unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < nseg;
        k += (unsigned long long)gridDim.x * blockDim.x) {
        const SegRec<double> &S = segs[k];
        if(S.job < 0) continue;
        const GroupDev &G = groups[find_group(groups, ngroups, S.job)];
        const Env3Dev &E = *G.env3;
        const bool gauss = E.gaussian != 0;
        const double freq = E.freq0;
        double sig = S.sigma_seg, fl = 0.0;
        if(gauss) {   // AdjustSigma (src/influence.hpp:91-100)
            fl = min(FLTD(0.2) * freq * S.tau1r, BHCB_PI * (S.c0 / freq));
            sig = max(sig, fl);
        }
        const double rmax = (gauss ? 4.0 : 1.0) * sig;
        const bool window = fabs(S.tx) > FLTD(0.50001);
        const int local = (int)((long long)S.job - G.job_base);
        const Job3 J = job_indices3(E, local);
        const long long plane = G.field_base
            + ((((long long)J.isz * E.nsx + J.isx) * E.nsy + J.isy) * E.ntheta + J.ibeta) * E.nrz * E.nrr;
        const float azim = (float)((180.0 / BHCB_PI) * E.beta[J.ibeta]);
        for(int iz = 0; iz < E.nrz; ++iz) {
            const double zr = (double)E.rz[iz];
            if(window && (zr < S.zlo - rmax || zr > S.zhi + rmax)) continue;
            const double dz = zr - S.x0z;
            for(int ir = S.ir_lo; ir <= S.ir_hi; ++ir) {
                const double dr = E.rr[ir] - S.x0r;
                const double s = (dr * S.tx + dz * S.tz) / S.rlen;
                const double n1 = fabs(dz * S.tx - dr * S.tz);
                const double qF = S.q0 + s * S.dq;
                double sigma = fabs(qF * S.rcp_q0);
                const double sig0 = sigma;
                if(gauss) sigma = max(sigma, fl);
                if(n1 >= (gauss ? 4.0 : 1.0) * sigma) continue;
                if(COUNT) {
                    ++count;
                    continue;
                }
                const unsigned long long i = atomicAdd(cursor, 1ull);
                if(i >= cand_cap) continue;
                if(kb.eigen) {
                    ArrCand c;
                    c.amp = c.phase = c.delay_re = c.delay_im = 0.0;
                    c.rcvr_decl = 0.f;
                    c.ntop = S.is;                   // step
                    c.nbot = ir;                     // receiver range
                    c.job = S.job;
                    c.aux = J.ibeta;                 // itheta = ibeta (src/influence.hpp:439)
                    c.rcvr_azim = __int_as_float(iz);
                    cands[i] = c;
                    const int walk = S.tx > 0.0 ? ir : E.nrr - 1 - ir;
                    const int gidx = (int)(&G - groups);
                    keys[i] = ((uint64_t)gidx << kb.sh_cell) | ((uint64_t)local << kb.sh_job)
                              | ((uint64_t)S.is << kb.sh_is) | ((uint64_t)walk << kb.sh_walk)
                              | ((uint64_t)J.ibeta << kb.sh_theta) | (uint64_t)iz;
                    vals[i] = (uint32_t)i;
                    continue;
                }
                const double w = gauss ? exp(FLTD(-0.5) * (n1 / sigma) * (n1 / sigma)) * (sig0 / sigma)
                                       : (sigma - n1) / sigma;
                const bool caustic = (qF <= 0.0 && S.q0 > 0.0) || (qF >= 0.0 && S.q0 < 0.0);
                const long long cell = plane + (long long)iz * E.nrr + ir;
                ArrCand c;
                c.amp = S.cnst_num / sqrt(fabs(qF)) * w;
                c.phase = caustic ? S.phase_b : S.phase_a;
                c.delay_re = S.tau0r + s * S.dtaur;
                c.delay_im = S.tau0i + s * S.dtaui;
                c.rcvr_decl = (float)S.rcvr_decl;
                c.rcvr_azim = azim;
                c.ntop = S.ntop;
                c.nbot = S.nbot;
                c.job = S.job;
                c.aux = J.ialpha;
                cands[i] = c;
                keys[i] = ((uint64_t)cell << kb.sh_cell) | ((uint64_t)local << kb.sh_job) | (uint64_t)S.is;
                vals[i] = (uint32_t)i;
            }
        }
    }
    if(COUNT && count) atomicAdd(&ctr->nevals, count);
}

// ScalePressure, 2-D form (src/influence.hpp:1556-1627): intensity to
// pressure for incoherent runs, then -1 / sqrt(r)
__global__ void scale_nx_kernel(float2 *field, const GroupDev *__restrict__ groups, int g)
{
    const GroupDev &G = groups[g];
    const Env3Dev &E = *G.env3;
    const long long n = (long long)E.nsz * E.nsx * E.nsy * E.ntheta * E.nrz * E.nrr;
    for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float2 u = field[G.field_base + i];
        if(!E.coherent) { u.x = sqrtf(u.x); u.y = 0.f; }
        const double r = E.rr[i % E.nrr];
        const double factor = fabs(r) < DBL_EPS ? 0.0 : FLTD(-1.0) / sqrt(fabs(r));
        const float ff = (float)factor;
        field[G.field_base + i] = make_float2(u.x * ff, u.y * ff);
    }
}

// Ray trajectories, Nx2D (MainRayMode, src/trace.hpp:485-519, with the
// points written in ocean coordinates as WriteRay does, src/mode/ray.hpp:
// 240-247): COUNT pass then fill pass as for the 2-D and 3-D rays.
template<bool COUNT>
__global__ void __launch_bounds__(64) ray_nx_kernel(const GroupDev *__restrict__ groups, int ngroups,
                                                    const long long *__restrict__ jobs, const int *__restrict__ limits,
                                                    int nitems, const long long *__restrict__ off, double *pts,
                                                    int *npts, int *bnc, RunCounters *ctr)
{
    for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < nitems; i += gridDim.x * blockDim.x) {
        const long long job = jobs[i];
        const GroupDev &G = groups[find_group(groups, ngroups, job)];
        const Env3Dev &E = *G.env3;
        const Job3 J = job_indices3(E, (int)(job - G.job_base));
        const int cap = COUNT ? 0x7fffffff : npts[i];
        const long long base = COUNT ? 0 : off[i];
        RayStateN st;
        auto put = [&](int idx, const RayN &p) {
            if(!COUNT && idx < cap) {
                const V3 x = to_ocean_x(p.x, st.org);
                double *q = pts + 3 * (base + idx);
                q[0] = x.x;
                q[1] = x.y;
                q[2] = x.z;
            }
        };
        if(J.isz >= E.nsz) {
            run_error(ctr, ERR_RAYINIT);
            if(COUNT) { npts[i] = 0; bnc[2 * i] = bnc[2 * i + 1] = 0; }
            continue;
        }
        int nsteps = -1, last_top = 0, last_bot = 0;
        if(!ray_init_nx(E, J, st, ctr)) {
            put(0, st.p0);
            nsteps = 1;
        } else {
            put(0, st.p0);
            const int limit = limits[i];
            int is = 0, small = 0, prev_top = 0, prev_bot = 0;
            RayN p1, p2;
            for(;;) {
                if((is & 31) == 0 && __ldcg(&ctr->err_bits) != 0u) {
                    nsteps = is + 1;
                    last_top = st.p0.ntop;
                    last_bot = st.p0.nbot;
                    break;
                }
                const bool two = ray_update_nx(st, p1, p2, small, E, ctr);
                put(is + 1, p1);
                if(two) put(is + 2, p2);
                if(limit >= 0 && is >= limit) {
                    nsteps = is + 2;
                    last_top = p1.ntop;
                    last_bot = p1.nbot;
                    break;
                }
                prev_top = two ? p1.ntop : st.p0.ntop;
                prev_bot = two ? p1.nbot : st.p0.nbot;
                is += two ? 2 : 1;
                st.p0 = two ? p2 : p1;
                if(ray_stops_nx(st, small, E)) {
                    nsteps = is + 1;
                    last_top = st.p0.ntop;
                    last_bot = st.p0.nbot;
                    break;
                }
                if(is >= MAXN_STEPS - 3) {
                    run_warn(ctr, WARN_ONERAY_OUTOFMEMORY);
                    nsteps = is;
                    last_top = prev_top;
                    last_bot = prev_bot;
                    break;
                }
            }
        }
        if(COUNT) {
            npts[i] = nsteps;
            bnc[2 * i] = last_top;
            bnc[2 * i + 1] = last_bot;
        }
    }
}

} // namespace

cudaError_t launch_rays_nx(const GroupDev *groups, int ngroups, const long long *jobs, const int *limits, int nitems,
                           const long long *off, double *pts, int *npts, int *bnc, RunCounters *ctr, bool count,
                           int sm_count, cudaStream_t st)
{
    if(nitems <= 0) return cudaSuccess;
    int grid = (nitems + 63) / 64;
    if(grid > sm_count * 16) grid = sm_count * 16;
    if(count)
        ray_nx_kernel<true><<<grid, 64, 0, st>>>(groups, ngroups, jobs, limits, nitems, off, pts, npts, bnc, ctr);
    else
        ray_nx_kernel<false><<<grid, 64, 0, st>>>(groups, ngroups, jobs, limits, nitems, off, pts, npts, bnc, ctr);
    return cudaGetLastError();
}

cudaError_t launch_trace_nx(const GroupDev *groups, int ngroups, long long job_end, void *segs,
                            unsigned long long cap, RunCounters *ctr, unsigned long long *job_counter, int grid,
                            cudaStream_t st)
{
    trace_nx_kernel<<<grid, 64, 0, st>>>(groups, ngroups, job_end, (SegRec<double> *)segs, cap, ctr, job_counter);
    return cudaGetLastError();
}

cudaError_t launch_arr_gather_nx(const void *segs, unsigned long long nseg, const GroupDev *groups, int ngroups,
                                 bool count, ArrCand *cands, uint64_t *keys, uint32_t *vals,
                                 unsigned long long cand_cap, unsigned long long *cursor, RunCounters *ctr,
                                 ArrKeyBits kb, int grid, cudaStream_t st)
{
    if(nseg == 0) return cudaSuccess;
    const SegRec<double> *S = (const SegRec<double> *)segs;
    if(count)
        arr_gather_nx_kernel<true><<<grid, 128, 0, st>>>(S, nseg, groups, ngroups, nullptr, nullptr, nullptr, 0,
                                                         nullptr, ctr, kb);
    else
        arr_gather_nx_kernel<false><<<grid, 128, 0, st>>>(S, nseg, groups, ngroups, cands, keys, vals, cand_cap,
                                                          cursor, ctr, kb);
    return cudaGetLastError();
}

cudaError_t launch_influence_nx(const void *segs, unsigned long long cap, const GroupDev *groups, int ngroups,
                                float2 *field, RunCounters *ctr, int nzmax, int grid, cudaStream_t st)
{
    if(nzmax < 1) nzmax = 1;
    influence_nx_kernel<<<grid, 128, 0, st>>>((const SegRec<double> *)segs, cap, groups, ngroups, field, ctr, nzmax);
    return cudaGetLastError();
}

cudaError_t launch_scale_nx(float2 *field, const GroupDev *groups, int g, int grid, cudaStream_t st)
{
    scale_nx_kernel<<<grid, 256, 0, st>>>(field, groups, g);
    return cudaGetLastError();
}

size_t nx_record_bytes() { return sizeof(SegRec<double>); }

} // namespace bhcb
