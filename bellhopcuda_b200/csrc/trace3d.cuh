// 3-D ray tracer device code (BELLHOP3D field modes, sm_100a, FP64).
//
// Restates, for the GPU, the per-ray physics of the reference's 3-D path:
// SSP evaluation (hexahedral src/ssp.hpp:215-305; 1-D profiles evaluated in
// depth, src/ssp.hpp:376-470), boundary cells of a triangulated grid
// (src/boundary.hpp:66-160), the modified-polygon step with 2x2 p-q dynamics,
// torsion and triangle-diagonal crossings (src/step.hpp:36-811), curvature
// corrections and reflection (src/step.hpp:478-627, src/reflect.hpp:125-452)
// and the ray driver (src/trace.hpp:51-589). The 2x2 matrices follow the GLM
// convention of the reference: m[column][row].
#pragma once
#include "bhcb_internal.h"
#include "device_math.cuh"
#include "trace2d.cuh"

#define DBL_MIN_POS 2.2250738585072014e-308   // smallest normal double (REAL_MINPOS)

namespace bhcb {

// ------------------------------------------------------------------ algebra
struct V3 {
    double x, y, z;
};
__device__ __forceinline__ V3 v3(double x, double y, double z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 add3(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 sub3(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 scl3(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross3(V3 u, V3 v)
{
    return {u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x};
}
__device__ __forceinline__ double len3(V3 a) { return sqrt(dot3(a, a)); }
__device__ __forceinline__ V3 ld3(const double *p) { return {p[0], p[1], p[2]}; }

struct M2 {
    double m[2][2];   // m[col][row]
};
__device__ __forceinline__ M2 m2_diag(double s)
{
    M2 r;
    r.m[0][0] = s; r.m[0][1] = 0.0; r.m[1][0] = 0.0; r.m[1][1] = s;
    return r;
}
// mat2x2(a, b, c, d): columns (a, b) and (c, d)
__device__ __forceinline__ M2 m2_cols(double a, double b, double c, double d)
{
    M2 r;
    r.m[0][0] = a; r.m[0][1] = b; r.m[1][0] = c; r.m[1][1] = d;
    return r;
}
__device__ __forceinline__ M2 m2_mul(const M2 &a, const M2 &b)
{
    M2 r;
    for(int c = 0; c < 2; ++c)
        for(int rr = 0; rr < 2; ++rr) r.m[c][rr] = a.m[0][rr] * b.m[c][0] + a.m[1][rr] * b.m[c][1];
    return r;
}
__device__ __forceinline__ M2 m2_T(const M2 &a)
{
    return m2_cols(a.m[0][0], a.m[1][0], a.m[0][1], a.m[1][1]);
}
__device__ __forceinline__ M2 m2_add(const M2 &a, const M2 &b)
{
    return m2_cols(a.m[0][0] + b.m[0][0], a.m[0][1] + b.m[0][1], a.m[1][0] + b.m[1][0], a.m[1][1] + b.m[1][1]);
}
__device__ __forceinline__ M2 m2_scl(double s, const M2 &a)
{
    return m2_cols(s * a.m[0][0], s * a.m[0][1], s * a.m[1][0], s * a.m[1][1]);
}
__device__ __forceinline__ double m2_det(const M2 &a) { return a.m[0][0] * a.m[1][1] - a.m[1][0] * a.m[0][1]; }
__device__ __forceinline__ bool nearly_zero(double x) { return fabs(x) < DBL_EPS; }

// ---------------------------------------------------------------------- SSP
struct SSPOut3 {
    V3 gradc;
    double c, ci, rho, cxx, cyy, czz, cxy, cxz, cyz;
};
struct Seg3 {
    int x, y, z;
};

// EvaluateSSP<O3D, R3D> (src/ssp.hpp:376-470)
template<bool NEED_RHO = false> __device__ __forceinline__ void eval_ssp3(
    V3 x, V3 t, SSPOut3 &o, const Env3Dev &E, Seg3 &s, RunCounters *ctr)
{
    o.cxx = o.cyy = o.cxy = o.cxz = o.cyz = 0.0;
    if(E.hex) {
        // Hexahedral (src/ssp.hpp:220-305)
        const int nx = E.hnx, ny = E.hny, nz = E.hnz;
        if(x.x < E.hx[0] || x.x > E.hx[nx - 1] || x.y < E.hy[0] || x.y > E.hy[ny - 1])
            run_error(ctr, ERR_OUTSIDE_SSP);
        update_seg(x.x, t.x >= 0.0, E.hx, nx, s.x);
        update_seg(x.y, t.y >= 0.0, E.hy, ny, s.y);
        update_seg(x.z, t.z >= 0.0, E.hz, nz, s.z);
        const int ix = s.x, iy = s.y, iz = s.z;
        const double cz11 = E.hcz[((size_t)ix * ny + iy) * (nz - 1) + iz];
        const double cz12 = E.hcz[((size_t)(ix + 1) * ny + iy) * (nz - 1) + iz];
        const double cz21 = E.hcz[((size_t)ix * ny + iy + 1) * (nz - 1) + iz];
        const double cz22 = E.hcz[((size_t)(ix + 1) * ny + iy + 1) * (nz - 1) + iz];
        double s3 = x.z - E.hz[iz];
        const double c11 = E.hc[((size_t)ix * ny + iy) * nz + iz] + s3 * cz11;
        const double c21 = E.hc[((size_t)(ix + 1) * ny + iy) * nz + iz] + s3 * cz12;
        const double c12 = E.hc[((size_t)ix * ny + iy + 1) * nz + iz] + s3 * cz21;
        const double c22 = E.hc[((size_t)(ix + 1) * ny + iy + 1) * nz + iz] + s3 * cz22;
        double s1 = (x.x - E.hx[ix]) / (E.hx[ix + 1] - E.hx[ix]);
        s1 = max(min(s1, 1.0), 0.0);
        double s2 = (x.y - E.hy[iy]) / (E.hy[iy + 1] - E.hy[iy]);
        s2 = max(min(s2, 1.0), 0.0);
        double c1 = c11 + s1 * (c21 - c11);
        double c2 = c12 + s1 * (c22 - c12);
        const double cy = (c2 - c1) / (E.hy[iy + 1] - E.hy[iy]);
        c1 = c11 + s2 * (c12 - c11);
        c2 = c21 + s2 * (c22 - c21);
        o.c = c1 + s1 * (c2 - c1);
        o.ci = 0.0;   // volume attenuation of the 1-D profile is not defined for 'H'
        const double cx = (c2 - c1) / (E.hx[ix + 1] - E.hx[ix]);
        const double cz1 = cz11 + s2 * (cz21 - cz11);
        const double cz2 = cz12 + s2 * (cz22 - cz12);
        o.gradc = v3(cx, cy, cz1 + s1 * (cz2 - cz1));
        o.czz = 0.0;
        // LinInterpDensity on the grid depths
        const double w = (x.z - E.e1d.z[iz]) / (E.e1d.z[iz + 1] - E.e1d.z[iz]);
        o.rho = (1.0 - w) * E.e1d.rho[iz] + w * E.e1d.rho[iz + 1];
        return;
    }
    // 1-D profile in depth
    SSPOut<double> o2;
    SegState s2{0, s.z};
    eval_ssp<double, NEED_RHO>(mk2(0.0, x.z), mk2(0.0, t.z), o2, E.e1d, s2, ctr);
    s.z = s2.z;
    o.gradc = v3(0.0, 0.0, o2.gradc.y);
    o.czz = o2.czz;
    o.c = o2.c;
    o.ci = o2.ci;
    o.rho = o2.rho;
}

// ----------------------------------------------------------------- boundary
struct Bd3 {
    int ix, iy;
    double xmin, xmax, ymin, ymax;   // cell limits
    V3 x, xmid, n;                   // corner node, cell centre, active triangle normal
    bool onEdge, side, justSteppedTo, outgoingSide;
};

// GetBdrySeg, 3-D branch (src/boundary.hpp:66-160)
__device__ __forceinline__ void get_bdry_seg3(V3 x, V3 t, Bd3 &b, const Bdry3PtDev *bd, int nx, int ny,
                                              bool istop, bool isinit, RunCounters *ctr)
{
    int ix = min(max(b.ix, 0), nx - 2);
    int iy = min(max(b.iy, 0), ny - 2);
    if(t.x >= 0.0) {
        while(ix >= 0 && bd[(size_t)ix * ny].x[0] > x.x) --ix;
        while(ix >= 0 && ix < nx - 1 && bd[(size_t)(ix + 1) * ny].x[0] <= x.x) ++ix;
    } else {
        while(ix < nx - 1 && bd[(size_t)(ix + 1) * ny].x[0] < x.x) ++ix;
        while(ix >= 0 && ix < nx - 1 && bd[(size_t)ix * ny].x[0] >= x.x) --ix;
    }
    if(t.y >= 0.0) {
        while(iy >= 0 && bd[iy].x[1] > x.y) --iy;
        while(iy >= 0 && iy < ny - 1 && bd[iy + 1].x[1] <= x.y) ++iy;
    } else {
        while(iy < ny - 1 && bd[iy + 1].x[1] < x.y) ++iy;
        while(iy >= 0 && iy < ny - 1 && bd[iy].x[1] >= x.y) --iy;
    }
    if(ix == -1 && bd[0].x[0] == x.x) ix = 0;
    if(ix == nx - 1 && bd[(size_t)(nx - 1) * ny].x[0] == x.x) ix = nx - 2;
    if(iy == -1 && bd[0].x[1] == x.y) iy = 0;
    if(iy == ny - 1 && bd[ny - 1].x[1] == x.y) iy = ny - 2;
    if(ix < 0 || ix >= nx - 1 || iy < 0 || iy >= ny - 1) {
        run_warn(ctr, istop ? WARN_OUTSIDE_ALTIMETRY : WARN_OUTSIDE_BATHYMETRY);
        ix = min(max(ix, 0), nx - 2);
        iy = min(max(iy, 0), ny - 2);
    }
    b.ix = ix;
    b.iy = iy;
    b.xmin = bd[(size_t)ix * ny].x[0];
    b.xmax = bd[(size_t)(ix + 1) * ny].x[0];
    b.ymin = bd[iy].x[1];
    b.ymax = bd[iy + 1].x[1];
    const Bdry3PtDev &p = bd[(size_t)ix * ny + iy];
    b.x = ld3(p.x);
    b.xmid = scl3(0.5, add3(b.x, ld3(bd[(size_t)(ix + 1) * ny + iy + 1].x)));
    // active triangle of the cell pair (normal of the diagonal, up and to the left)
    double tnx = -(b.ymax - b.ymin), tny = b.xmax - b.xmin;
    const double tl = sqrt(tnx * tnx + tny * tny);
    tnx /= tl;
    tny /= tl;
    const double over = (x.x - b.xmid.x) * tnx + (x.y - b.xmid.y) * tny;
    b.onEdge = fabs(over) < 3e-6;   // TRIDIAG_THRESH (FP64)
    if(!isinit && b.justSteppedTo) b.side = b.outgoingSide;
    else if(!isinit && b.onEdge) b.side = (t.x * tnx + t.y * tny) >= 0.0;
    else b.side = over >= 0.0;
    b.justSteppedTo = false;
    b.n = b.side ? ld3(p.n2) : ld3(p.n1);
    if(!isfinite(b.x.z) || !isfinite(b.n.x) || !isfinite(b.n.y) || !isfinite(b.n.z))
        run_error(ctr, ERR_BOUNDARY_SEG_NAN);
}

// Distances (src/trace.hpp:37-45)
__device__ __forceinline__ void distances3(V3 x, const Bd3 &top, const Bd3 &bot, double &dt, double &db)
{
    dt = -dot3(top.n, sub3(x, top.x));
    db = -dot3(bot.n, sub3(x, bot.x));
}


// --------------------------------------------------------------- ray state
struct Ray3 {
    V3 x, t;
    M2 p, q;
    double c, Amp, Phase, phi, taur, taui;
    int ntop, nbot;
};

// RayNormalImpl (src/common_run.hpp:144-199)
__device__ __forceinline__ void ray_normal(V3 t, double phi, bool ignorephi0, double c, V3 &e1, V3 &e2)
{
    const double rl = sqrt(t.x * t.x + t.y * t.y);
    if(!nearly_zero(phi) || ignorephi0) {
        const double cp = cos(phi), sp = sin(phi);
        e1.x = (c * t.x * t.z * cp + t.y * sp) / rl;
        e1.y = (c * t.y * t.z * cp - t.x * sp) / rl;
        e1.z = -c * rl * cp;
        e2.x = (c * t.x * t.z * sp - t.y * cp) / rl;
        e2.y = (c * t.y * t.z * sp + t.x * cp) / rl;
        e2.z = -c * rl * sp;
    } else {
        e1 = v3(c * t.x * t.z / rl, c * t.y * t.z / rl, -c * rl);
        e2 = v3(-t.y / rl, t.x / rl, 0.0);
    }
}

// CalcTangent_Normals (src/step.hpp:566-576)
__device__ __forceinline__ void tangent_normals(const Ray3 &r, double c, V3 nB, V3 &rayt, V3 &rayn1, V3 &rayn2,
                                                double sign2)
{
    rayt = scl3(c, r.t);
    rayn2 = scl3(sign2, cross3(rayt, nB));
    rayn2 = scl3(1.0 / len3(rayn2), rayn2);
    rayn1 = scl3(-1.0, cross3(rayt, rayn2));
}

// ------------------------------------------------------------ step geometry
// src/step.hpp:41-79 (depth interfaces; none past the first / last layer in 3-D)
__device__ __forceinline__ void depth_iface3(bool stepTo, double &h, V3 &x, V3 x0, V3 u, int iz0, const Env3Dev &E,
                                             int &snap)
{
    if(!stepTo) h = 1.7976931348623157e308;
    if(fabs(u.z) > DBL_EPS) {
        const double *z = E.e1d.z;
        const int nz = E.e1d.nssp;
        if(z[iz0] > x.z && iz0 > 0) {
            h = (z[iz0] - x0.z) / u.z;
            if(stepTo) { x = add3(x0, scl3(h, u)); x.z = z[iz0]; snap = 2; }
        } else if(z[iz0 + 1] < x.z && iz0 + 1 < nz - 1) {
            h = (z[iz0 + 1] - x0.z) / u.z;
            if(stepTo) { x = add3(x0, scl3(h, u)); x.z = z[iz0 + 1]; snap = 2; }
        }
    }
}

__device__ __forceinline__ double comp3(V3 v, int d) { return d == 0 ? v.x : (d == 1 ? v.y : v.z); }
__device__ __forceinline__ void setc3(V3 &v, int d, double a)
{
    if(d == 0) v.x = a; else if(d == 1) v.y = a; else v.z = a;
}

// BeamBoxCrossing (src/step.hpp:84-108): box centred at (source x, y, 0)
__device__ __forceinline__ void box3(bool stepTo, int d, double &h, V3 &x, V3 x0, V3 u, V3 xs, const Env3Dev &E,
                                     int &snap)
{
    if(!stepTo) h = 1.7976931348623157e308;
    const double bx = d == 0 ? E.box_x : (d == 1 ? E.box_y : E.box_z);
    const double ctr = d == 2 ? 0.0 : comp3(xs, d);
    if(fabs(comp3(x, d) - ctr) >= bx) {
        const double d0 = comp3(x0, d) - ctr;
        h = (bx - fabs(d0)) / fabs(comp3(u, d));
        if(stepTo) {
            x = add3(x0, scl3(h, u));
            setc3(x, d, ctr + copysign(bx, d0));
            snap = d;
        }
    }
}

// TopBotCrossing (src/step.hpp:113-147)
__device__ __forceinline__ void topbot3(bool stepTo, double &h, const Bd3 &bd, V3 &x, V3 x0, V3 u, bool &refl,
                                        int &snap)
{
    if(!stepTo) h = 1.7976931348623157e308;
    const V3 d = sub3(x, bd.x), d0 = sub3(x0, bd.x);
    const double w = dot3(bd.n, d);
    if(stepTo ? (w > -INF_STEP) : (w >= 0.0)) {
        h = -dot3(d0, bd.n) / dot3(u, bd.n);
        if(stepTo) {
            x = add3(x0, scl3(h, u));
            if(fabs(bd.n.x) < DBL_EPS && fabs(bd.n.y) < DBL_EPS) x.z = bd.x.z;
            snap = 2;   // exactness in depth matters most, flat or not
        }
        refl = true;
    } else {
        refl = false;
    }
}

// TopBotSegCrossing in x or y (src/step.hpp:153-205), with the hexahedral cell limits
__device__ __forceinline__ void cellseg3(bool stepTo, bool isY, double &h, const Bd3 &top, const Bd3 &bot, V3 &x,
                                         V3 x0, V3 u, const Env3Dev &E, const Seg3 &s0, bool &tr, bool &br, int &snap)
{
    double lmin = isY ? max(top.ymin, bot.ymin) : max(top.xmin, bot.xmin);
    double lmax = isY ? min(top.ymax, bot.ymax) : min(top.xmax, bot.xmax);
    if(E.hex) {
        const double *w = isY ? E.hy : E.hx;
        const int i = isY ? s0.y : s0.x;
        lmin = max(lmin, w[i]);
        lmax = min(lmax, w[i + 1]);
    }
    const double xw = isY ? x.y : x.x, x0w = isY ? x0.y : x0.x, uw = isY ? u.y : u.x;
    if(!stepTo) h = 1.7976931348623157e308;
    if(fabs(uw) > DBL_EPS) {
        if(xw < lmin) {
            h = -(x0w - lmin) / uw;
            if(stepTo) {
                x = add3(x0, scl3(h, u));
                if(isY) x.y = lmin; else x.x = lmin;
                snap = isY ? 1 : 0;
                tr = br = false;
            }
        } else if(xw > lmax) {
            h = -(x0w - lmax) / uw;
            if(stepTo) {
                x = add3(x0, scl3(h, u));
                if(isY) x.y = lmax; else x.x = lmax;
                snap = isY ? 1 : 0;
                tr = br = false;
            }
        }
    }
}

// TriDiagCrossing (src/step.hpp:210-256)
__device__ __forceinline__ void tridiag3(bool stepTo, double &h, Bd3 &bd, V3 &x, V3 x0, V3 u, bool &tr, bool &br,
                                         RunCounters *ctr, int &snap)
{
    if(!stepTo) h = 1.7976931348623157e308;
    if(bd.onEdge) return;
    const V3 d = sub3(x, bd.xmid), d0 = sub3(x0, bd.xmid);
    V3 tn = v3(-(bd.ymax - bd.ymin), bd.xmax - bd.xmin, 0.0);
    tn = scl3(1.0 / len3(tn), tn);
    const double over = dot3(d, tn);
    const bool newSide = over >= 0.0;
    if(newSide == bd.side) return;
    if(fabs(over) < 3e-6) return;   // stepped right onto the edge
    const double hnew = -dot3(d0, tn) / dot3(u, tn);
    if(hnew < 0.0) {
        run_warn(ctr, WARN_TRIDIAG_H_NEGATIVE);
        h = 0.0;
    } else {
        if(stepTo && hnew >= h) run_warn(ctr, WARN_TRIDIAG_H_GROWING);
        h = hnew;
    }
    if(stepTo) {
        x = add3(x0, scl3(h, u));
        bd.justSteppedTo = true;
        bd.outgoingSide = newSide;
        snap = -2;   // x or y, unspecified
        tr = br = false;
    }
}

// ReduceStep, 3-D (src/step.hpp:265-340)
__device__ __forceinline__ void reduce_step3(V3 x0, V3 u, const Seg3 &s0, Bd3 &top, Bd3 &bot, V3 xs,
                                             const Env3Dev &E, double &h, int &small, RunCounters *ctr)
{
    double hInt, hB0, hB1, hB2, hTop, hBot, hX, hY, hTD, hBD;
    bool dummy = false, d2 = false;
    int sn = -1;
    V3 x = add3(x0, scl3(h, u));
    depth_iface3(false, hInt, x, x0, u, s0.z, E, sn);
    box3(false, 0, hB0, x, x0, u, xs, E, sn);
    box3(false, 1, hB1, x, x0, u, xs, E, sn);
    box3(false, 2, hB2, x, x0, u, xs, E, sn);
    topbot3(false, hTop, top, x, x0, u, dummy, sn);
    topbot3(false, hBot, bot, x, x0, u, dummy, sn);
    cellseg3(false, false, hX, top, bot, x, x0, u, E, s0, dummy, d2, sn);
    cellseg3(false, true, hY, top, bot, x, x0, u, E, s0, dummy, d2, sn);
    tridiag3(false, hTD, top, x, x0, u, dummy, d2, ctr, sn);
    tridiag3(false, hBD, bot, x, x0, u, dummy, d2, ctr, sn);
    h = min(min(min(h, hInt), min(min(min(hB0, hB1), hB2), min(hTop, hBot))), min(min(hX, hY), min(hTD, hBD)));
    if(h < -1e-4) run_warn(ctr, WARN_STEP_NEGATIVE_H);
    const double hmin = INF_STEP * E.deltas;
    if(h < hmin) {
        h = hmin;
        ++small;
    } else {
        small = 0;
    }
}

// StepToBdry, 3-D (src/step.hpp:345-422); snap: the coordinate the landing
// point was put on exactly (OceanToRayX's snapDim: -1 none, 0 x, 1 y, 2 z,
// -2 x or y)
__device__ __forceinline__ void step_to_bdry3(V3 x0, V3 &x2, V3 u, double &h, bool &tr, bool &br, const Seg3 &s0,
                                              Bd3 &top, Bd3 &bot, V3 xs, const Env3Dev &E, RunCounters *ctr, int &snap)
{
    x2 = add3(x0, scl3(h, u));
    snap = -1;
    depth_iface3(true, h, x2, x0, u, s0.z, E, snap);
    box3(true, 0, h, x2, x0, u, xs, E, snap);
    box3(true, 1, h, x2, x0, u, xs, E, snap);
    box3(true, 2, h, x2, x0, u, xs, E, snap);
    topbot3(true, h, top, x2, x0, u, tr, snap);
    topbot3(true, h, bot, x2, x0, u, br, snap);
    if(br) tr = false;
    cellseg3(true, false, h, top, bot, x2, x0, u, E, s0, tr, br, snap);
    cellseg3(true, true, h, top, bot, x2, x0, u, E, s0, tr, br, snap);
    tridiag3(true, h, top, x2, x0, u, tr, br, ctr, snap);
    tridiag3(true, h, bot, x2, x0, u, tr, br, ctr, snap);
    const double hmin = INF_STEP * E.deltas;
    if(h < hmin) {
        h = hmin;
        x2 = add3(x0, scl3(h, u));
        snap = -1;
        if(dot3(top.n, sub3(x2, top.x)) > DBL_EPS) {
            tr = true;
            top.justSteppedTo = false;
            bot.justSteppedTo = false;
            snap = 2;
        } else {
            tr = false;
        }
        if(dot3(bot.n, sub3(x2, bot.x)) > DBL_EPS) {
            br = true;
            tr = false;
            top.justSteppedTo = false;
            bot.justSteppedTo = false;
            snap = 2;
        } else {
            br = false;
        }
    }
}


// ---------------------------------------------------------------- dynamics
struct Part3 {
    double cnn, cmn, cmm;
};
struct DPQ3 {
    double phi;
    M2 p, q;
};

// Get_c_partials, 3-D (src/step.hpp:425-446)
__device__ __forceinline__ Part3 c_partials3(const Ray3 &r, const SSPOut3 &o)
{
    V3 e1, e2;
    ray_normal(r.t, r.phi, false, o.c, e1, e2);
    Part3 q;
    q.cnn = o.cxx * e1.x * e1.x + o.cyy * e1.y * e1.y + o.czz * e1.z * e1.z + 2.0 * o.cxy * e1.x * e1.y
        + 2.0 * o.cxz * e1.x * e1.z + 2.0 * o.cyz * e1.y * e1.z;
    q.cmn = o.cxx * e1.x * e2.x + o.cyy * e1.y * e2.y + o.czz * e1.z * e2.z + o.cxy * (e1.x * e2.y + e2.x * e1.y)
        + o.cxz * (e1.x * e2.z + e2.x * e1.z) + o.cyz * (e1.y * e2.z + e2.y * e1.z);
    q.cmm = o.cxx * e2.x * e2.x + o.cyy * e2.y * e2.y + o.czz * e2.z * e2.z + 2.0 * o.cxy * e2.x * e2.y
        + 2.0 * o.cxz * e2.x * e2.z + 2.0 * o.cyz * e2.y * e2.z;
    return q;
}

// ComputeDeltaPQ, 3-D (src/step.hpp:448-468): torsion rate, p' = q C^T, q' = c p
__device__ __forceinline__ DPQ3 delta_pq3(const Ray3 &r, const SSPOut3 &o, const Part3 &pt)
{
    DPQ3 d;
    d.phi = (1.0 / o.c) * r.t.z * (r.t.y * o.gradc.x - r.t.x * o.gradc.y) / (r.t.x * r.t.x + r.t.y * r.t.y);
    M2 cm = m2_scl(-1.0 / (o.c * o.c), m2_cols(pt.cnn, pt.cmn, pt.cmn, pt.cmm));
    d.p = m2_mul(r.q, m2_T(cm));
    d.q = m2_scl(o.c, r.p);
    return d;
}

// UpdateRayPQ (src/step.hpp:470-476)
__device__ __forceinline__ void update_pq3(Ray3 &r1, const Ray3 &r0, double h, const DPQ3 &d)
{
    r1.phi = r0.phi + h * d.phi;
    r1.p = m2_add(r0.p, m2_scl(h, d.p));
    r1.q = m2_add(r0.q, m2_scl(h, d.q));
}

// CurvatureCorrection3D<REFLECT> (src/step.hpp:483-564)
template<bool REFLECT> __device__ __forceinline__ void curv_corr3(
    Ray3 &r, const M2 &D, double Tg, double Th, double cn1j, double cn2j, double csj, V3 rayn1, V3 rayn2,
    V3 e1, V3 e2)
{
    const double rm = Tg / Th;
    const double csq = r.c * r.c;
    M2 R;
    R.m[0][0] = 2.0 / csq * D.m[0][0] / Th + rm * (2.0 * cn1j - rm * csj) / csq;
    R.m[0][1] = 2.0 / r.c * D.m[1][0] * copysign(1.0, -Th) + rm * cn2j / csq;
    R.m[1][0] = R.m[0][1];
    R.m[1][1] = 2.0 * D.m[1][1] * Th;
    if(REFLECT) R.m[1][0] = -R.m[1][0];
    else R = m2_scl(-1.0, R);
    bool nochange = false;
    if(REFLECT) nochange = nearly_zero(R.m[0][0]) && nearly_zero(R.m[0][1]) && nearly_zero(R.m[1][1]);
    if(!nochange) {
        M2 Rot;
        Rot.m[0][0] = dot3(rayn1, e1);
        Rot.m[1][0] = dot3(rayn1, e2);
        Rot.m[0][1] = -Rot.m[1][0];
        Rot.m[1][1] = dot3(rayn2, e2);
        const M2 pin = m2_mul(Rot, r.p);
        const M2 qin = m2_mul(Rot, r.q);
        const M2 pout = m2_add(pin, m2_mul(R, qin));
        r.p = m2_mul(m2_T(Rot), pout);
    }
    if(REFLECT) {
        const double d = dot3(rayn1, e1);
        r.phi += 2.0 * acos(max(min(d, 1.0), -1.0));
    }
}

// CurvatureCorrection, 3-D (src/step.hpp:581-621): jump in the sound-speed
// gradient across an SSP cell face
__device__ __forceinline__ void interface_corr3(Ray3 &r, V3 gradcjump, const Seg3 &s, const Seg3 &s0)
{
    V3 nB = v3(0.0, 0.0, 0.0);
    if(s.z != s0.z) nB.z = -copysign(1.0, r.t.z);
    else if(s.x != s0.x) nB.x = -copysign(1.0, r.t.x);
    else nB.y = -copysign(1.0, r.t.y);
    const double Th = dot3(r.t, nB);
    V3 tB = sub3(r.t, scl3(Th, nB));
    tB = scl3(1.0 / len3(tB), tB);
    const double Tg = dot3(r.t, tB);
    V3 rayt, rayn1, rayn2, e1, e2;
    tangent_normals(r, r.c, nB, rayt, rayn1, rayn2, 1.0);
    ray_normal(rayt, r.phi, true, 1.0, e1, e2);
    const double cn1j = dot3(gradcjump, rayn1), cn2j = dot3(gradcjump, rayn2), csj = dot3(gradcjump, rayt);
    curv_corr3<false>(r, m2_diag(0.0), Tg, Th, cn1j, cn2j, csj, rayn1, rayn2, e1, e2);
}

// Step, 3-D (src/step.hpp:654-811): modified polygon method with step
// reduction onto interfaces, cell faces, triangle diagonals and the beam box
__device__ __forceinline__ void step3d(const Ray3 &r0, Ray3 &r2, Bd3 &top, Bd3 &bot, V3 xs, const Env3Dev &E,
                                       Seg3 &iSeg, int &small, bool &tr, bool &br, RunCounters *ctr)
{
    SSPOut3 o0, o1, o2;
    eval_ssp3(r0.x, r0.t, o0, E, iSeg, ctr);
    const DPQ3 d0 = delta_pq3(r0, o0, c_partials3(r0, o0));
    const Seg3 s0 = iSeg;
    const double csq0 = o0.c * o0.c;
    const V3 u0 = scl3(o0.c, r0.t);
    double h = E.deltas;
    reduce_step3(r0.x, u0, s0, top, bot, xs, E, h, small, ctr);
    const double halfh = 0.5 * h;
    Ray3 r1;
    r1.x = add3(r0.x, scl3(halfh, u0));
    r1.t = sub3(r0.t, v3(halfh * o0.gradc.x / csq0, halfh * o0.gradc.y / csq0, halfh * o0.gradc.z / csq0));
    update_pq3(r1, r0, halfh, d0);

    eval_ssp3(r1.x, r1.t, o1, E, iSeg, ctr);
    const DPQ3 d1 = delta_pq3(r1, o1, c_partials3(r1, o1));
    const double csq1 = o1.c * o1.c;
    const V3 u1 = scl3(o1.c, r1.t);
    reduce_step3(r0.x, u1, s0, top, bot, xs, E, h, small, ctr);
    const double w1 = h / (2.0 * halfh);
    const double w0 = 1.0 - w1;
    const V3 u2 = add3(scl3(w0, u0), scl3(w1, u1));
    int snap;
    step_to_bdry3(r0.x, r2.x, u2, h, tr, br, s0, top, bot, xs, E, ctr, snap);
    const double hw0 = h * w0, hw1 = h * w1;
    r2.t = v3(r0.t.x - hw0 * o0.gradc.x / csq0 - hw1 * o1.gradc.x / csq1,
              r0.t.y - hw0 * o0.gradc.y / csq0 - hw1 * o1.gradc.y / csq1,
              r0.t.z - hw0 * o0.gradc.z / csq0 - hw1 * o1.gradc.z / csq1);
    const Cx<double> a0 = o0.ci == 0.0 ? cx<double>(hw0 / o0.c, 0.0) : rdivc(hw0, cx<double>(o0.c, o0.ci));
    const Cx<double> a1 = o1.ci == 0.0 ? cx<double>(hw1 / o1.c, 0.0) : rdivc(hw1, cx<double>(o1.c, o1.ci));
    r2.taur = r0.taur + a0.r + a1.r;
    r2.taui = r0.taui + a0.i + a1.i;
    update_pq3(r2, r0, hw0, d0);
    update_pq3(r2, r2, hw1, d1);
    r2.Amp = r0.Amp;
    r2.Phase = r0.Phase;
    r2.ntop = r0.ntop;
    r2.nbot = r0.nbot;
    eval_ssp3(r2.x, r2.t, o2, E, iSeg, ctr);
    r2.c = o2.c;
    if(iSeg.z != s0.z || iSeg.x != s0.x || iSeg.y != s0.y)
        interface_corr3(r2, sub3(o2.gradc, o0.gradc), iSeg, s0);
}

// Reflect, 3-D (src/reflect.hpp:125-452): nB the boundary normal (a
// triangle's, or interpolated between the node normals of a curvilinear
// grid), zxx, zxy, zyy the cell's depth curvatures (0 for flat triangles);
// the halfspace uses the gamma form
__device__ __forceinline__ void reflect3d(const Ray3 &old, Ray3 &np, const HsDev &hs, bool istop, V3 nB,
                                          double zxx, double zxy, double zyy, const Env3Dev &E, Seg3 &iSeg,
                                          RunCounters *ctr)
{
    const double Th = dot3(old.t, nB);
    V3 tB = sub3(old.t, scl3(Th, nB));
    tB = scl3(1.0 / len3(tB), tB);
    const double Tg = dot3(old.t, tB);
    np.ntop = old.ntop + (istop ? 1 : 0);
    np.nbot = old.nbot + (istop ? 0 : 1);
    np.x = old.x;
    np.t = sub3(old.t, scl3(2.0 * Th, nB));
    SSPOut3 o;
    eval_ssp3<true>(old.x, np.t, o, E, iSeg, ctr);
    np.c = o.c;
    np.taur = old.taur;
    np.taui = old.taui;
    V3 rayt, rayn1, rayn2, rayt_t, rayn1_t, rayn2_t;
    tangent_normals(old, o.c, nB, rayt, rayn1, rayn2, -1.0);
    tangent_normals(np, o.c, nB, rayt_t, rayn1_t, rayn2_t, -1.0);
    // DMat = Rot^T (2 kappa) Rot, kappa = [[zxx, zxy], [zxy, zyy]] / 2
    double tx = rayt.x, ty = rayt.y;
    double tl = sqrt(tx * tx + ty * ty);
    tx /= tl; ty /= tl;
    double nx = rayn2.x, ny = rayn2.y;
    double nl = sqrt(nx * nx + ny * ny);
    nx /= nl; ny /= nl;
    const M2 Rot = m2_cols(tx, ty, nx, ny);
    const M2 K2 = m2_cols(FLTD(2.0) * (zxx / FLTD(2.0)), FLTD(2.0) * (zxy / FLTD(2.0)), FLTD(2.0) * (zxy / FLTD(2.0)),
                          FLTD(2.0) * (zyy / FLTD(2.0)));
    const M2 D = m2_mul(m2_T(Rot), m2_mul(K2, Rot));
    const double cn1j = dot3(o.gradc, sub3(scl3(-1.0, rayn1_t), rayn1));
    const double cn2j = dot3(o.gradc, sub3(scl3(-1.0, rayn2_t), rayn2));
    const double csj = -dot3(o.gradc, sub3(rayt_t, rayt));
    V3 e1, e2;
    ray_normal(old.t, old.phi, false, old.c, e1, e2);
    np.p = old.p;
    np.q = old.q;
    np.phi = old.phi;
    curv_corr3<true>(np, D, Tg, Th, cn1j, cn2j, csj, rayn1, rayn2, e1, e2);

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
    } else if(hs.bc == 'A' || hs.bc == 'G') {
        const double omega = FLTD(2.0) * BHCB_PI * E.freq0;
        const double gk = omega * Tg;
        const double wc = omega / o.c;
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


// GetJobIndices, 3-D (src/common.hpp:365-391): ialpha fastest, then ibeta, isy, isx, isz
struct Job3 {
    int ialpha, ibeta, isx, isy, isz;
};
__device__ __forceinline__ Job3 job_indices3(const Env3Dev &E, int local)
{
    Job3 j;
    if(E.isingle_alpha >= 1) {
        j.ialpha = E.isingle_alpha - 1;
    } else {
        j.ialpha = local % E.nalpha;
        local /= E.nalpha;
    }
    if(E.isingle_beta >= 1) {
        j.ibeta = E.isingle_beta - 1;
    } else {
        j.ibeta = local % E.nbeta;
        local /= E.nbeta;
    }
    j.isy = local % E.nsy;
    local /= E.nsy;
    j.isx = local % E.nsx;
    local /= E.nsx;
    j.isz = local;
    return j;
}

} // namespace bhcb
