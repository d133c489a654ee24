// 3-D ray driver shared by the BELLHOP3D kernels: per-ray state, RayInit,
// RayUpdate and RayTerminate's stop conditions (src/trace.hpp:76-477).
#pragma once
#include "bhcb_internal.h"
#include "device_math.cuh"
#include "trace2d.cuh"
#include "influence2d.cuh"
#include "trace3d.cuh"

namespace bhcb {

// Per-ray state of the 3-D ray loop.
struct RayState3 {
    Ray3 p0;
    Bd3 top, bot;
    Seg3 iSeg;
    V3 xs;
    double alpha, beta, c;
    double minx, miny, maxx, maxy;   // extent of the boundary grids (RayTerminate)
};

// RayInit (src/trace.hpp:76-266), 3-D: false when the source is on or outside
// the boundaries (the ray is not traced)
__device__ __forceinline__ bool ray_init3d(const Env3Dev &E, const Job3 &J, RayState3 &st, RunCounters *ctr)
{
    const double alpha = E.alpha[J.ialpha], beta = E.beta[J.ibeta];
    st.alpha = alpha;
    st.beta = beta;
    const double SrcDecl = (180.0 / BHCB_PI) * alpha;
    st.iSeg = Seg3{0, 0, 0};
    const V3 xs = v3(E.sx[J.isx], E.sy[J.isy], (double)E.sz[J.isz]);
    st.xs = xs;
    SSPOut3 o;
    eval_ssp3(xs, v3(0.0, 0.0, 1.0), o, E, st.iSeg, ctr);
    const double c = o.c;
    st.c = c;
    const int ibp = min(bsearch_leq2(E.sbp, E.nsbp, SrcDecl), E.nsbp - 2);
    const double s = (SrcDecl - E.sbp[2 * ibp]) / (E.sbp[2 * (ibp + 1)] - E.sbp[2 * ibp]);
    float amp0 = (float)((FLTD(1.0) - s) * E.sbp[2 * ibp + 1] + s * E.sbp[2 * (ibp + 1) + 1]);
    if(E.run0 == 'S') {
        const float om = (float)(FLTD(2.0) * BHCB_PI * E.freq0);
        amp0 = (float)(amp0 * ((double)sqrtf(2.0f) * fabs(sin(om / c * xs.z * sin(alpha)))));
    }
    Ray3 &p0 = st.p0;
    // launch direction from the host's cos / sin of the angles (the reference's RayInit computes them on the CPU)
    const double ca = E.acs[2 * J.ialpha], sa = E.acs[2 * J.ialpha + 1];
    const V3 tinit = v3(ca * E.bcs[2 * J.ibeta], ca * E.bcs[2 * J.ibeta + 1], sa);
    p0.x = xs;
    p0.c = c;
    p0.t = v3(tinit.x / c, tinit.y / c, tinit.z / c);
    p0.taur = p0.taui = 0.0;
    p0.Amp = (double)amp0;
    p0.Phase = 0.0;
    p0.ntop = p0.nbot = 0;
    p0.p = m2_diag(1.0);
    p0.q = m2_diag(0.0);
    p0.phi = 0.0;
    st.top.ix = st.top.iy = st.bot.ix = st.bot.iy = 0;
    st.top.justSteppedTo = st.bot.justSteppedTo = false;
    st.top.side = st.bot.side = false;
    st.top.outgoingSide = st.bot.outgoingSide = false;
    get_bdry_seg3(xs, p0.t, st.top, E.btop, E.top_nx, E.top_ny, true, true, ctr);
    get_bdry_seg3(xs, p0.t, st.bot, E.bbot, E.bot_nx, E.bot_ny, false, true, ctr);
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

// RayUpdate (src/trace.hpp:274-381), 3-D: one step from st.p0 to p1 and, on a
// boundary hit, the reflected point p2; returns whether p2 was produced
__device__ __forceinline__ bool ray_update3d(RayState3 &st, Ray3 &p1, Ray3 &p2, int &small, const Env3Dev &E,
                                             RunCounters *ctr)
{
    bool tr = false, br = false;
    step3d(st.p0, p1, st.top, st.bot, st.xs, E, st.iSeg, small, tr, br, ctr);
    get_bdry_seg3(p1.x, p1.t, st.top, E.btop, E.top_nx, E.top_ny, true, false, ctr);
    get_bdry_seg3(p1.x, p1.t, st.bot, E.bbot, E.bot_nx, E.bot_ny, false, false, ctr);
    const bool two = tr || br;
    if(two) {
        const Bd3 &b = tr ? st.top : st.bot;
        V3 nI = b.n;
        double zxx = 0.0, zxy = 0.0, zyy = 0.0;
        if(tr ? E.top_curv : E.bot_curv) {
            // curvilinear grid: normal interpolated between the cell's node
            // normals, curvature of the cell (src/trace.hpp:318-341)
            const Bdry3PtDev *bd = tr ? E.btop : E.bbot;
            const int ny = tr ? E.top_ny : E.bot_ny;
            const double s1 = (p1.x.x - b.x.x) / (b.xmax - b.xmin), s2 = (p1.x.y - b.x.y) / (b.ymax - b.ymin);
            const double m1 = 1.0 - s1, m2 = 1.0 - s2;
            const Bdry3PtDev &d00 = bd[(size_t)b.ix * ny + b.iy], &d01 = bd[(size_t)b.ix * ny + b.iy + 1];
            const Bdry3PtDev &d10 = bd[(size_t)(b.ix + 1) * ny + b.iy], &d11 = bd[(size_t)(b.ix + 1) * ny + b.iy + 1];
            nI = v3(d00.noden[0] * m1 * m2 + d10.noden[0] * s1 * m2 + d11.noden[0] * s1 * s2 + d01.noden[0] * m1 * s2,
                    d00.noden[1] * m1 * m2 + d10.noden[1] * s1 * m2 + d11.noden[1] * s1 * s2 + d01.noden[1] * m1 * s2,
                    d00.noden[2] * m1 * m2 + d10.noden[2] * s1 * m2 + d11.noden[2] * s1 * s2 + d01.noden[2] * m1 * s2);
            zxx = d00.zxx;
            zxy = d00.zxy;
            zyy = d00.zyy;
        }
        reflect3d(p1, p2, tr ? E.top : E.bot, tr, nI, zxx, zxy, zyy, E, st.iSeg, ctr);
    }
    return two;
}

// RayTerminate's stop conditions (src/trace.hpp:391-477), 3-D
__device__ __forceinline__ bool ray_stops3d(const RayState3 &st, int small, const Env3Dev &E)
{
    const V3 x = st.p0.x, t = st.p0.t;
    const bool leftbox = fabs(x.x - st.xs.x) >= E.box_x || fabs(x.y - st.xs.y) >= E.box_y || fabs(x.z) >= E.box_z;
    const bool esc0 = x.x < st.minx || x.y < st.miny || (x.x == st.minx && t.x < 0.0) || (x.y == st.miny && t.y < 0.0);
    const bool escN = x.x > st.maxx || x.y > st.maxy || (x.x == st.maxx && t.x > 0.0) || (x.y == st.maxy && t.y > 0.0);
    const bool lost = st.p0.Amp < FLTD(0.005);
    return leftbox || lost || esc0 || escN || small > 50;
}

} // namespace bhcb
