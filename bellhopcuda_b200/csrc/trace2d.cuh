// 2-D ray tracer device code (sm_100a).
//
// Restates, for the GPU, the per-ray physics of the reference's field modes:
// SSP evaluation (src/ssp.hpp:36-465), boundary segment tracking
// (src/boundary.hpp:66-227), the modified-polygon step with boundary-landing
// step reduction (src/step.hpp:41-811), reflection (src/reflect.hpp:125-452)
// and the ray driver (src/trace.hpp:76-589). Template parameter R is the bulk
// arithmetic type: double for the FP64 tracer, float for the mixed tracer.
// In both, positions, the travel-time accumulation and the step-length /
// boundary-crossing solves are FP64, so rays land on the same interfaces.
#pragma once
#include "bhcb_internal.h"
#include "device_math.cuh"

namespace bhcb {

#define BHCB_PI 3.14159265358979323846
#define INF_STEP 1e-6       // src/step.hpp:28-32
#define MAXN_STEPS 100000   // include/bhc/structs.hpp:66
#define DBL_EPS 2.220446049250313e-16
#define FLTD(x) ((double)(x##f))   // reference FL() literals are float

template<typename R> struct SSPOut {
    V2<R> gradc;
    R c, ci, rho, czz, crr, crz;
};

struct SegState { int r, z; };

struct BdState {
    int Iseg;
    double lmin, lmax;
    V2<double> x, n;
};

template<typename R> struct RayPt {
    int ntop, nbot;
    V2<double> x;
    V2<R> t, p, q;
    R c, Amp, Phase;
    double taur, taui;
};

__device__ __forceinline__ void run_error(RunCounters *ctr, int code)
{
    atomicOr(&ctr->err_bits, 1u << code);
}
__device__ __forceinline__ void run_warn(RunCounters *ctr, int code)
{
    if(!(__ldcg(&ctr->warn_bits) & (1u << code))) atomicOr(&ctr->warn_bits, 1u << code);
}

// src/ssp.hpp:36-51 — direction-aware segment walk
__device__ __forceinline__ void update_seg(double x, bool tpos, const double *a, int n, int &iSeg)
{
    if(tpos) {
        while(iSeg > 0 && x < a[iSeg]) --iSeg;
        while(iSeg < n - 2 && x >= a[iSeg + 1]) ++iSeg;
    } else {
        while(iSeg < n - 2 && x > a[iSeg + 1]) ++iSeg;
        while(iSeg > 0 && x <= a[iSeg]) --iSeg;
    }
}

// src/ssp.hpp:157-212 — quad (range-dependent) SSP: bilinear in range between
// two profiles, each linear in depth; the attenuation comes from the .env
// profile. The density is always interpolated (LinInterpDensity).
template<typename R> __device__ __forceinline__ void eval_quad(
    V2<double> x, V2<R> t, SSPOut<R> &o, const EnvDev &e, SegState &s, RunCounters *ctr)
{
    const int nr = e.nqr;
    if(x.x < e.qr[0] || x.x > e.qr[nr - 1]) run_error(ctr, ERR_OUTSIDE_SSP);
    update_seg(x.y, t.y >= (R)0, e.z, e.nssp, s.z);
    update_seg(x.x, t.x >= (R)0, e.qr, nr, s.r);
    {
        double z0 = e.z[s.z];
        R w = (R)((x.y - z0) / (e.z[s.z + 1] - z0));
        o.rho = ((R)1 - w) * (R)e.rho[s.z] + w * (R)e.rho[s.z + 1];
    }
    if(s.z >= e.nssp - 1 || s.r >= nr - 1) {
        run_error(ctr, ERR_QUAD_ISEG);
        s.z = s.r = 0;
    }
    const int iz = s.z, ir = s.r;
    const R cz1 = (R)e.qcz[iz * nr + ir], cz2 = (R)e.qcz[iz * nr + ir + 1];
    const double s2d = x.y - e.z[iz];
    const R s2 = (R)s2d;
    const R dz = (R)(e.z[iz + 1] - e.z[iz]);
    const R c1 = (R)e.qc[iz * nr + ir] + s2 * cz1;
    const R c2 = (R)e.qc[iz * nr + ir + 1] + s2 * cz2;
    const R dr = (R)(e.qr[ir + 1] - e.qr[ir]);
    R s1 = (R)(x.x - e.qr[ir]) / dr;
    s1 = min(s1, (R)1);
    s1 = max(s1, (R)0);
    o.c = ((R)1 - s1) * c1 + s1 * c2;
    const R w2 = s2 / dz;
    o.ci = ((R)1 - w2) * (R)e.c[2 * iz + 1] + w2 * (R)e.c[2 * iz + 3];
    const R cz = ((R)1 - s1) * cz1 + s1 * cz2;
    o.gradc = mk2<R>((c2 - c1) / dr, cz);
    o.crz = (cz2 - cz1) / dr;
}

// src/ssp.hpp:53-152,309-375 (1-D profile types evaluated in 2-D). The
// density (LinInterpDensity) is only used by reflections, so it is evaluated
// when NEED_RHO is set.
template<typename R, bool NEED_RHO = false> __device__ __forceinline__ void eval_ssp(
    V2<double> x, V2<R> t, SSPOut<R> &o, const EnvDev &e, SegState &s, RunCounters *ctr)
{
    o.crr = o.crz = o.czz = (R)0;
    if(e.ssp_type == SSP_ANALYTIC) {
        s.z = 0;
        const R c0 = (R)1500.0, u1 = (R)FLTD(1300.0), u2 = (R)FLTD(0.00737);
        o.rho = (R)1;
        R xt = (R)2 * ((R)x.y - u1) / u1;
        R emxt = exp(-xt);
        R dxt = (R)2 / u1;
        o.c = c0 * ((R)1 + u2 * (xt - (R)1 + emxt));
        o.ci = (R)0;
        o.gradc = mk2<R>((R)0, c0 * u2 * ((R)1 - emxt) * dxt);
        o.czz = c0 * u2 * emxt * dxt * dxt;
        return;
    }
    if(e.ssp_type == SSP_QUAD) {
        eval_quad(x, t, o, e, s, ctr);
        return;
    }
    update_seg(x.y, t.y >= (R)0, e.z, e.nssp, s.z);
    int iz = s.z;
    double z0 = e.z[iz];
    double dz = x.y - z0;
    R w = (R)0;
    if(NEED_RHO || e.ssp_type == SSP_N2LINEAR) {
        w = (R)(dz / (e.z[iz + 1] - z0));
        o.rho = ((R)1 - w) * (R)e.rho[iz] + w * (R)e.rho[iz + 1];
    } else {
        o.rho = (R)0;
    }
    switch(e.ssp_type) {
    case SSP_CLINEAR: {
        o.c = (R)e.c[2 * iz] + (R)dz * (R)e.cz[2 * iz];
        o.ci = (R)e.c[2 * iz + 1] + (R)dz * (R)e.cz[2 * iz + 1];
        o.gradc = mk2<R>((R)0, (R)e.cz[2 * iz]);
    } break;
    case SSP_N2LINEAR: {
        Cx<R> n2 = cadd(cscl((R)1 - w, cx<R>((R)e.n2[2 * iz], (R)e.n2[2 * iz + 1])),
                        cscl(w, cx<R>((R)e.n2[2 * iz + 2], (R)e.n2[2 * iz + 3])));
        Cx<R> cc = rdivc((R)1, csqrt_(n2));
        o.c = cc.r;
        o.ci = cc.i;
        R c = cc.r;
        o.gradc = mk2<R>((R)0, (R)-0.5 * (c * c * c) * (R)e.n2z[2 * iz]);
        o.czz = (R)3 * o.gradc.y * o.gradc.y / c;
    } break;
    case SSP_CUBIC: {
        // SplineALL (src/curves.hpp:190-204)
        const double *C = e.coef;
        int n = e.nssp;
        R h = (R)dz;
        R c1r = (R)C[2 * iz], c1i = (R)C[2 * iz + 1];
        R c2r = (R)C[2 * (n + iz)], c2i = (R)C[2 * (n + iz) + 1];
        R c3r = (R)C[2 * (2 * n + iz)], c3i = (R)C[2 * (2 * n + iz) + 1];
        R c4r = (R)C[2 * (3 * n + iz)], c4i = (R)C[2 * (3 * n + iz) + 1];
        const R half = (R)0.5, sixth = (R)(double)(1.0f / 6.0f);
        o.c = c1r + h * (c2r + h * (half * c3r + sixth * h * c4r));
        o.ci = c1i + h * (c2i + h * (half * c3i + sixth * h * c4i));
        o.gradc = mk2<R>((R)0, c2r + h * (c3r + h * half * c4r));
        o.czz = c3r + h * c4r;
    } break;
    case SSP_PCHIP: {
        const double *C = e.coef;
        int n = e.nssp;
        R xt = (R)dz;
        R a0 = (R)C[2 * iz], a0i = (R)C[2 * iz + 1];
        R a1 = (R)C[2 * (n + iz)], a1i = (R)C[2 * (n + iz) + 1];
        R a2 = (R)C[2 * (2 * n + iz)], a2i = (R)C[2 * (2 * n + iz) + 1];
        R a3 = (R)C[2 * (3 * n + iz)], a3i = (R)C[2 * (3 * n + iz) + 1];
        o.c = a0 + (a1 + (a2 + a3 * xt) * xt) * xt;
        o.ci = a0i + (a1i + (a2i + a3i * xt) * xt) * xt;
        o.gradc = mk2<R>((R)0, a1 + ((R)2 * a2 + (R)3 * a3 * xt) * xt);
        o.czz = (R)2 * a2 + (R)6 * a3 * xt;
    } break;
    default: run_error(ctr, ERR_INVALID_SSP_TYPE);
    }
}

// Register copy of the SSP segment a ray is in, for the 1-D profile types
// C, S and P: the segment's depth bounds and its coefficients, reloaded only
// when update_seg would move the segment. It holds the table values
// themselves and eval_ssp_cached does eval_ssp's arithmetic on them, so the
// results are the same; it saves the dependent table loads of every
// evaluation on the ray's step chain.
struct SspSegCache {
    int type;          // e.ssp_type; other types take eval_ssp
    int iz;            // segment held (-1: none)
    bool down, up;     // update_seg may move the segment down / up from iz
    double z0, z1;     // e.z[iz], e.z[iz + 1]
    double k0, k1, k2, k3, k4, k5, k6, k7;   // C: c, cz (re, im); S, P: the four complex coefficients
};

__device__ __forceinline__ void ssp_cache_init(SspSegCache &sc, const EnvDev &e)
{
    sc.type = e.ssp_type;
    sc.iz = -1;
}

template<typename R> __device__ __forceinline__ void eval_ssp_cached(
    V2<double> x, V2<R> t, SSPOut<R> &o, const EnvDev &e, SegState &s, SspSegCache &sc, RunCounters *ctr)
{
    if(sc.type != SSP_CLINEAR && sc.type != SSP_CUBIC && sc.type != SSP_PCHIP) {
        eval_ssp(x, t, o, e, s, ctr);
        return;
    }
    const bool tpos = t.y >= (R)0;
    // the segment update_seg would leave unchanged (src/ssp.hpp:36-51)
    bool move = sc.iz != s.z;
    if(!move)
        move = tpos ? ((sc.down && x.y < sc.z0) || (sc.up && x.y >= sc.z1))
                    : ((sc.up && x.y > sc.z1) || (sc.down && x.y <= sc.z0));
    if(move) {
        const int n = e.nssp;
        update_seg(x.y, tpos, e.z, n, s.z);
        const int iz = s.z;
        sc.iz = iz;
        sc.down = iz > 0;
        sc.up = iz < n - 2;
        sc.z0 = e.z[iz];
        sc.z1 = e.z[iz + 1];
        if(sc.type == SSP_CLINEAR) {
            sc.k0 = e.c[2 * iz];
            sc.k1 = e.c[2 * iz + 1];
            sc.k2 = e.cz[2 * iz];
            sc.k3 = e.cz[2 * iz + 1];
        } else {
            const double *C = e.coef;
            sc.k0 = C[2 * iz];
            sc.k1 = C[2 * iz + 1];
            sc.k2 = C[2 * (n + iz)];
            sc.k3 = C[2 * (n + iz) + 1];
            sc.k4 = C[2 * (2 * n + iz)];
            sc.k5 = C[2 * (2 * n + iz) + 1];
            sc.k6 = C[2 * (3 * n + iz)];
            sc.k7 = C[2 * (3 * n + iz) + 1];
        }
    }
    const double dz = x.y - sc.z0;
    o.crr = o.crz = o.czz = (R)0;
    o.rho = (R)0;
    if(sc.type == SSP_CLINEAR) {
        o.c = (R)sc.k0 + (R)dz * (R)sc.k2;
        o.ci = (R)sc.k1 + (R)dz * (R)sc.k3;
        o.gradc = mk2<R>((R)0, (R)sc.k2);
    } else if(sc.type == SSP_CUBIC) {
        // SplineALL (src/curves.hpp:190-204)
        const R h = (R)dz;
        const R c1r = (R)sc.k0, c1i = (R)sc.k1, c2r = (R)sc.k2, c2i = (R)sc.k3;
        const R c3r = (R)sc.k4, c3i = (R)sc.k5, c4r = (R)sc.k6, c4i = (R)sc.k7;
        const R half = (R)0.5, sixth = (R)(double)(1.0f / 6.0f);
        o.c = c1r + h * (c2r + h * (half * c3r + sixth * h * c4r));
        o.ci = c1i + h * (c2i + h * (half * c3i + sixth * h * c4i));
        o.gradc = mk2<R>((R)0, c2r + h * (c3r + h * half * c4r));
        o.czz = c3r + h * c4r;
    } else {
        const R xt = (R)dz;
        const R a0 = (R)sc.k0, a0i = (R)sc.k1, a1 = (R)sc.k2, a1i = (R)sc.k3;
        const R a2 = (R)sc.k4, a2i = (R)sc.k5, a3 = (R)sc.k6, a3i = (R)sc.k7;
        o.c = a0 + (a1 + (a2 + a3 * xt) * xt) * xt;
        o.ci = a0i + (a1i + (a2i + a3i * xt) * xt) * xt;
        o.gradc = mk2<R>((R)0, a1 + ((R)2 * a2 + (R)3 * a3 * xt) * xt);
        o.czz = (R)2 * a2 + (R)6 * a3 * xt;
    }
}

// src/boundary.hpp:66-227 (2-D branch)
__device__ __forceinline__ void get_bdry_seg(
    V2<double> x, double tx, BdState &bs, const BdryPtDev *bd, int n, bool islong, HsDev &hs,
    bool istop, bool isinit, RunCounters *ctr)
{
    if(!isinit
       && !(x.x < bs.lmin || (x.x == bs.lmin && tx < 0.0) || x.x > bs.lmax
            || (x.x == bs.lmax && tx >= 0.0)))
        return;
    int is = min(max(bs.Iseg, 0), n - 2);
    if(tx >= 0.0) {
        while(is >= 0 && bd[is].x[0] > x.x) --is;
        while(is >= 0 && is < n - 1 && bd[is + 1].x[0] <= x.x) ++is;
    } else {
        while(is < n - 1 && bd[is + 1].x[0] < x.x) ++is;
        while(is >= 0 && is < n - 1 && bd[is].x[0] >= x.x) --is;
    }
    if(is < 0 || is >= n - 1) {
        run_error(ctr, istop ? ERR_OUTSIDE_ALTIMETRY : ERR_OUTSIDE_BATHYMETRY);
        is = 0;
    }
    bs.Iseg = is;
    bs.lmin = bd[is].x[0];
    bs.lmax = bd[is + 1].x[0];
    bs.x = mk2(bd[is].x[0], bd[is].x[1]);
    bs.n = mk2(bd[is].n[0], bd[is].n[1]);
    if(islong) {
        hs.cPr = bd[is].cPr; hs.cPi = bd[is].cPi;
        hs.cSr = bd[is].cSr; hs.cSi = bd[is].cSi;
        hs.rho = bd[is].rho;
    }
}

// src/trace.hpp:37-45
__device__ __forceinline__ void distances(
    V2<double> x, const BdState &top, const BdState &bot, double &dt, double &db)
{
    dt = -dot2(top.n, sub2(x, top.x));
    db = -dot2(bot.n, sub2(x, bot.x));
}

__device__ __forceinline__ double dimv(V2<double> v, int d) { return d == 0 ? v.x : v.y; }

// src/step.hpp:41-79 (depth interface), 84-108 (beam box), 113-147 (top/bottom),
// 153-205 (range segment); all solves in FP64
struct StepGeo {
    const EnvDev *e;
    __device__ __forceinline__ void depth_iface(bool stepTo, double &h, V2<double> &x, V2<double> x0,
                                                V2<double> u, int iz0) const
    {
        if(!stepTo) h = 1.7976931348623157e308;
        if(fabs(u.y) > DBL_EPS) {
            double za = e->z[iz0], zb = e->z[iz0 + 1];
            if(za > x.y) {
                h = (za - x0.y) / u.y;
                if(stepTo) { x = add2(x0, scl2(h, u)); x.y = za; }
            } else if(zb < x.y) {
                h = (zb - x0.y) / u.y;
                if(stepTo) { x = add2(x0, scl2(h, u)); x.y = zb; }
            }
        }
    }
    __device__ __forceinline__ void box(bool stepTo, int d, double &h, V2<double> &x, V2<double> x0,
                                        V2<double> u) const
    {
        if(!stepTo) h = 1.7976931348623157e308;
        double bx = d == 0 ? e->box_x : e->box_y;
        if(fabs(dimv(x, d)) >= bx) {
            double d0 = dimv(x0, d);
            h = (bx - fabs(d0)) / fabs(dimv(u, d));
            if(stepTo) {
                x = add2(x0, scl2(h, u));
                if(d == 0) x.x = copysign(bx, d0); else x.y = copysign(bx, d0);
            }
        }
    }
    __device__ __forceinline__ void topbot(bool stepTo, double &h, const BdState &bd, V2<double> &x,
                                           V2<double> x0, V2<double> u, bool &refl) const
    {
        if(!stepTo) h = 1.7976931348623157e308;
        V2<double> d = sub2(x, bd.x), d0 = sub2(x0, bd.x);
        double w = dot2(bd.n, d);
        if(stepTo ? (w > -INF_STEP) : (w >= 0.0)) {
            h = -dot2(d0, bd.n) / dot2(u, bd.n);
            if(stepTo) {
                x = add2(x0, scl2(h, u));
                if(fabs(bd.n.x) < DBL_EPS) x.y = bd.x.y;
            }
            refl = true;
        } else {
            refl = false;
        }
    }
    __device__ __forceinline__ void seg(bool stepTo, double &h, const BdState &top, const BdState &bot,
                                        V2<double> &x, V2<double> x0, V2<double> u, bool &tr,
                                        bool &br, int ir0) const
    {
        double lmin = max(top.lmin, bot.lmin), lmax = min(top.lmax, bot.lmax);
        if(e->ssp_type == SSP_QUAD) {          // the quad SSP's range segment bounds the step too
            lmin = max(lmin, e->qr[ir0]);
            lmax = min(lmax, e->qr[ir0 + 1]);
        }
        if(!stepTo) h = 1.7976931348623157e308;
        if(fabs(u.x) > DBL_EPS) {
            if(x.x < lmin) {
                h = -(x0.x - lmin) / u.x;
                if(stepTo) { x = add2(x0, scl2(h, u)); x.x = lmin; tr = br = false; }
            } else if(x.x > lmax) {
                h = -(x0.x - lmax) / u.x;
                if(stepTo) { x = add2(x0, scl2(h, u)); x.x = lmax; tr = br = false; }
            }
        }
    }
};

// src/step.hpp:271-342
__device__ __forceinline__ void reduce_step(
    const StepGeo &g, V2<double> x0, V2<double> u, SegState s0, const BdState &top, const BdState &bot,
    double &h, int &small, RunCounters *ctr)
{
    double hInt, hB0, hB1, hTop, hBot, hSeg;
    bool dummy;
    V2<double> x = add2(x0, scl2(h, u));
    g.depth_iface(false, hInt, x, x0, u, s0.z);
    g.box(false, 0, hB0, x, x0, u);
    g.box(false, 1, hB1, x, x0, u);
    g.topbot(false, hTop, top, x, x0, u, dummy);
    g.topbot(false, hBot, bot, x, x0, u, dummy);
    g.seg(false, hSeg, top, bot, x, x0, u, dummy, dummy, s0.r);
    h = min(min(min(h, hInt), min(min(hB0, hB1), min(hTop, hBot))), hSeg);
    if(h < -1e-4) run_warn(ctr, WARN_STEP_NEGATIVE_H);
    double hmin = INF_STEP * g.e->deltas;
    if(h < hmin) {
        h = hmin;
        ++small;
    } else {
        small = 0;
    }
}

// src/step.hpp:347-424
__device__ __forceinline__ void step_to_bdry(
    const StepGeo &g, V2<double> x0, V2<double> &x2, V2<double> u, double &h, bool &tr, bool &br,
    SegState s0, const BdState &top, const BdState &bot)
{
    x2 = add2(x0, scl2(h, u));
    g.depth_iface(true, h, x2, x0, u, s0.z);
    g.box(true, 0, h, x2, x0, u);
    g.box(true, 1, h, x2, x0, u);
    g.topbot(true, h, top, x2, x0, u, tr);
    g.topbot(true, h, bot, x2, x0, u, br);
    if(br) tr = false;
    g.seg(true, h, top, bot, x2, x0, u, tr, br, s0.r);
    double hmin = INF_STEP * g.e->deltas;
    if(h < hmin) {
        h = hmin;
        x2 = add2(x0, scl2(h, u));
        tr = dot2(top.n, sub2(x2, top.x)) > DBL_EPS;
        br = dot2(bot.n, sub2(x2, bot.x)) > DBL_EPS;
        if(br) tr = false;
    }
}

// src/step.hpp:654-811 (2-D), with src/step.hpp:426-478 (p-q dynamics) and
// src/step.hpp:589-649 (interface curvature correction)
template<typename R> __device__ __forceinline__ void step2d(
    const RayPt<R> &ray0, RayPt<R> &ray2, const BdState &top, const BdState &bot,
    const EnvDev &e, SegState &iSeg, int &small, bool &tr, bool &br, RunCounters *ctr,
    SspSegCache *sc = nullptr)
{
    StepGeo g{&e};
    SSPOut<R> o0, o1, o2;
#define BHCB_STEP_SSP(X, T, O) \
    do { if(sc) eval_ssp_cached(X, T, O, e, iSeg, *sc, ctr); else eval_ssp(X, T, O, e, iSeg, ctr); } while(0)
    BHCB_STEP_SSP(ray0.x, ray0.t, o0);
    R cnn0 = o0.crr * ray0.t.y * ray0.t.y - (R)2 * o0.crz * ray0.t.x * ray0.t.y
        + o0.czz * ray0.t.x * ray0.t.x;
    V2<R> pq0p = scl2(-cnn0, ray0.q), pq0q = scl2(o0.c, ray0.p);
    SegState s0 = iSeg;
    R csq0 = o0.c * o0.c;
    V2<R> u0 = scl2(o0.c, ray0.t);
    double h = e.deltas;
    reduce_step(g, ray0.x, cvt2<double>(u0), s0, top, bot, h, small, ctr);
    double halfh = 0.5 * h;
    RayPt<R> ray1;
    ray1.x = add2(ray0.x, scl2(halfh, cvt2<double>(u0)));
    ray1.t = sub2(ray0.t, div2(scl2((R)halfh, o0.gradc), csq0));
    ray1.p = add2(ray0.p, scl2((R)halfh, pq0p));
    ray1.q = add2(ray0.q, scl2((R)halfh, pq0q));

    BHCB_STEP_SSP(ray1.x, ray1.t, o1);
    R cnn1 = o1.crr * ray1.t.y * ray1.t.y - (R)2 * o1.crz * ray1.t.x * ray1.t.y
        + o1.czz * ray1.t.x * ray1.t.x;
    V2<R> pq1p = scl2(-cnn1, ray1.q), pq1q = scl2(o1.c, ray1.p);
    R csq1 = o1.c * o1.c;
    V2<R> u1 = scl2(o1.c, ray1.t);
    reduce_step(g, ray0.x, cvt2<double>(u1), s0, top, bot, h, small, ctr);
    double w1 = h / (2.0 * halfh);
    double w0 = 1.0 - w1;
    V2<double> u2 = add2(scl2(w0, cvt2<double>(u0)), scl2(w1, cvt2<double>(u1)));
    step_to_bdry(g, ray0.x, ray2.x, u2, h, tr, br, s0, top, bot);
    double hw0 = h * w0, hw1 = h * w1;
    ray2.t = sub2(sub2(ray0.t, div2(scl2((R)hw0, o0.gradc), csq0)), div2(scl2((R)hw1, o1.gradc), csq1));
    // travel time in FP64: tau += hw0 / c0 + hw1 / c1 (complex sound speed)
    // (a real divisor is divided directly; cdiv gives the same value for it)
    Cx<double> d0 = o0.ci == (R)0 ? cx<double>(hw0 / (double)o0.c, 0.0)
                                  : rdivc(hw0, cx<double>((double)o0.c, (double)o0.ci));
    Cx<double> d1 = o1.ci == (R)0 ? cx<double>(hw1 / (double)o1.c, 0.0)
                                  : rdivc(hw1, cx<double>((double)o1.c, (double)o1.ci));
    ray2.taur = ray0.taur + d0.r + d1.r;
    ray2.taui = ray0.taui + d0.i + d1.i;
    ray2.p = add2(add2(ray0.p, scl2((R)hw0, pq0p)), scl2((R)hw1, pq1p));
    ray2.q = add2(add2(ray0.q, scl2((R)hw0, pq0q)), scl2((R)hw1, pq1q));
    ray2.Amp = ray0.Amp;
    ray2.Phase = ray0.Phase;
    ray2.ntop = ray0.ntop;
    ray2.nbot = ray0.nbot;
    BHCB_STEP_SSP(ray2.x, ray2.t, o2);
#undef BHCB_STEP_SSP
    ray2.c = o2.c;
    if(iSeg.z != s0.z || iSeg.r != s0.r) {
        // iSeg.r only moves for the quad SSP; a depth crossing takes precedence
        V2<R> gj = sub2(o2.gradc, o0.gradc);
        V2<R> n2 = mk2(-ray2.t.y, ray2.t.x);
        R cnj = dot2(gj, n2), csj = dot2(gj, ray2.t);
        R rm = iSeg.z != s0.z ? ray2.t.x / ray2.t.y : -ray2.t.y / ray2.t.x;
        R rn = rm * ((R)2 * cnj - rm * csj) / ray2.c;
        ray2.p = sub2(ray2.p, scl2(rn, ray2.q));
    }
}

// InterpolateReflectionCoefficient (src/reflect.hpp:39-92): linear in the
// angle of incidence theta (deg) between bracketing table rows; zero outside
// the table (a warning below it). A one-row table matches only its own angle.
template<typename R> __device__ __forceinline__ void refl_coef(const double *tab, int n, R theta, R &r, R &phi,
                                                              RunCounters *ctr)
{
    if(theta < (R)tab[0]) {
        r = phi = (R)0;
        run_warn(ctr, WARN_OUTSIDE_REFLCOEF);
        return;
    }
    if(theta > (R)tab[3 * (n - 1)]) {
        r = phi = (R)0;
        return;
    }
    if(n < 2) {
        r = (R)tab[1];
        phi = (R)tab[2];
        return;
    }
    int il = 0, ir = n - 1;
    while(ir - il > 1) {
        int im = (il + ir) >> 1;
        if((R)tab[3 * im] > theta) ir = im; else il = im;
    }
    const R t0 = (R)tab[3 * il], t1 = (R)tab[3 * ir];
    const R a = (theta - t0) / (t1 - t0);
    r = ((R)1 - a) * (R)tab[3 * il + 1] + a * (R)tab[3 * ir + 1];
    phi = ((R)1 - a) * (R)tab[3 * il + 2] + a * (R)tab[3 * ir + 2];
}

// Beam displacement and width change on a halfspace reflection (RunType(7)
// 'S'; src/reflect.hpp:383-448, Tindle's formulas as the reference states
// them): the reflected point moves along the boundary tangent by Re(delta),
// the travel time grows by Re(delta) cos / c, and q by |d delta| sin c p.
template<typename R> __device__ __forceinline__ void beam_shift2d(const RayPt<R> &old, RayPt<R> &np,
                                                                  const HsDev &hs, V2<R> tB, R omega, R c)
{
    const Cx<R> cPc = cx<R>((R)hs.cPr, -(R)hs.cPi);                 // conj(cP)
    const Cx<R> ch = rdivc(old.c, cPc);
    const R co = old.t.x * old.c, si = old.t.y * old.c;
    const R ck = omega / old.c;
    const R rho = (R)hs.rho;
    const Cx<R> one_m_ch2 = csub(cx<R>((R)1, (R)0), cmul(ch, ch));
    const Cx<R> a = cscl((R)2 * rho, one_m_ch2);
    const Cx<R> b = csub(cx<R>(co * co, (R)0), cmul(ch, ch));
    const Cx<R> d = cadd(cx<R>(rho * rho * si * si, (R)0), b);
    const Cx<R> sb = csqrt_(b);
    const R cco = co * co, ssi = si * si;
    Cx<R> delta = cx<R>((R)0, (R)0);
    if(fabs(si) >= (R)DBL_EPS)                                     // NotNearlyZero
        delta = cdiv(cscl(co / si, a), cscl(ck, cmul(sb, d)));
    const R pdelta = delta.r / (old.c / co);
    const Cx<R> cksbd = cscl(ck, cmul(sb, d));
    const Cx<R> t1 = rdivc(cco, cmul(cksbd, b));
    const Cx<R> t2 = rdivc((R)1 + cco / ssi, cksbd);
    const Cx<R> t3 = rdivc((R)2 * co * co * (rho * rho - (R)1), cmul(cksbd, d));
    const Cx<R> dd = cmul(a, csub(csub(t1, t2), t3));
    const R rdd = -dd.r;
    const R sdd = rdd / fabs(rdd);
    const R theta_bot = atan(tB.y / tB.x);
    np.x.x = np.x.x + (double)(delta.r * cos(theta_bot));
    np.x.y = np.x.y + (double)(delta.r * sin(theta_bot));
    np.taur = np.taur + (double)pdelta;
    np.q = add2(np.q, scl2(sdd * rdd * si * c, old.p));
}

// src/reflect.hpp:125-452 (2-D branch)
template<typename R> __device__ __forceinline__ void reflect2d(
    const RayPt<R> &old, RayPt<R> &np, const HsDev &hs, bool istop, V2<R> tB, V2<R> nB, R kappa,
    const EnvDev &e, SegState &iSeg, RunCounters *ctr)
{
    R Th = dot2(old.t, nB);
    R Tg = dot2(old.t, tB);
    np.ntop = old.ntop + (istop ? 1 : 0);
    np.nbot = old.nbot + (istop ? 0 : 1);
    np.x = old.x;
    np.t = sub2(old.t, scl2((R)2 * Th, nB));
    SSPOut<R> o;
    eval_ssp<R, true>(old.x, old.t, o, e, iSeg, ctr);
    R c = o.c;
    np.c = c;
    np.taur = old.taur;
    np.taui = old.taui;
    V2<R> rayt = scl2(c, old.t), rayn = mk2(-rayt.y, rayt.x);
    V2<R> rayt_t = scl2(c, np.t), rayn_t = mk2(rayt_t.y, -rayt_t.x);
    R rn = (R)2 * kappa / (c * c) / Th;
    R cnjump = -dot2(o.gradc, sub2(rayn_t, rayn));
    R csjump = -dot2(o.gradc, sub2(rayt_t, rayt));
    if(istop) { cnjump = -cnjump; rn = -rn; }
    R rm = Tg / Th;
    rn += rm * ((R)2 * cnjump - rm * csjump) / (c * c);
    if(e.beam2 == 'D') rn *= (R)2;
    else if(e.beam2 == 'Z') rn = (R)0;
    np.p = add2(old.p, scl2(rn, old.q));
    np.q = old.q;
    if(hs.bc == 'R') {
        np.Amp = old.Amp;
        np.Phase = old.Phase;
    } else if(hs.bc == 'V') {
        np.Amp = old.Amp;
        np.Phase = old.Phase + (R)BHCB_PI;
    } else if(hs.bc == 'F') {
        // angle of incidence from the boundary normal, folded about 90 deg
        R theta = (R)(180.0 / BHCB_PI) * fabs(atan2(Th, Tg));
        if(theta > (R)90) theta = (R)180 - theta;
        R rc, ph;
        refl_coef(istop ? e.trc : e.brc, istop ? e.ntrc : e.nbrc, theta, rc, ph, ctr);
        np.Amp = old.Amp * rc;
        np.Phase = old.Phase + ph;
    } else if(hs.bc == 'A' || hs.bc == 'G') {
        R omega = (R)(2.0 * BHCB_PI * e.freq0);
        Cx<R> kx = cx<R>(omega * Tg, (R)0), kz = cx<R>(omega * Th, (R)0);
        Cx<R> kx2 = cmul(kx, kx);
        Cx<R> cP = cx<R>((R)hs.cPr, (R)hs.cPi), cS = cx<R>((R)hs.cSr, (R)hs.cSi);
        Cx<R> f, gg;
        if(cS.r > (R)0) {
            Cx<R> wS = rdivc(omega, cS), wP = rdivc(omega, cP);
            Cx<R> kzS2 = csub(kx2, cmul(wS, wS)), kzP2 = csub(kx2, cmul(wP, wP));
            Cx<R> kzS = csqrt_(kzS2), kzP = csqrt_(kzP2);
            Cx<R> mu = cscl((R)hs.rho, cmul(cS, cS));
            Cx<R> a = cadd(kzS2, kx2);
            Cx<R> y2 = cmul(csub(cmul(a, a), cscl((R)4, cmul(cmul(kzS, kzP), kx2))), mu);
            Cx<R> y4 = cmul(kzP, csub(kx2, kzS2));
            f = cscl(omega * omega, y4);
            gg = y2;
        } else {
            Cx<R> wP = rdivc(omega, cP);
            Cx<R> kzP = csqrt_(csub(kx2, cmul(wP, wP)));
            if(fabs(kzP.r) < (R)DBL_EPS && kzP.i < (R)0) { kzP.r = -kzP.r; kzP.i = -kzP.i; }
            f = kzP;
            gg = cx<R>((R)hs.rho, (R)0);
        }
        Cx<R> rf = cscl(o.rho, f);
        Cx<R> jkg = cmul(cx<R>(-kz.i, kz.r), gg);     // J * kz * g
        Cx<R> num = csub(rf, jkg), den = cadd(rf, jkg);
        Cx<R> Refl = cdiv(num, den);
        Refl.r = -Refl.r;
        Refl.i = -Refl.i;
        R ar = cabs_(Refl);
        if(ar < (R)FLTD(1.0e-5)) {
            np.Amp = (R)0;
            np.Phase = old.Phase;
        } else {
            np.Amp = ar * old.Amp;
            np.Phase = old.Phase + atan2(Refl.i, Refl.r);
            if(e.beam_shift) beam_shift2d(old, np, hs, tB, omega, c);
        }
    } else {
        run_error(ctr, ERR_BOUNDARY_CONDITION_TYPE);
        np.Amp = (R)NAN;
        np.Phase = (R)NAN;
    }
}

} // namespace bhcb
