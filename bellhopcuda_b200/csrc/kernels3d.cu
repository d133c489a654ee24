// 3-D (BELLHOP3D) field-mode kernels for sm_100a, FP64.
//
//  trace3d_kernel     one ray per thread (persistent, work-queue driven):
//                     RayInit / RayUpdate / RayTerminate of the 3-D path
//                     (src/trace.hpp:76-477) and the sequential part of
//                     Step_InfluenceGeoCart's 3-D branch (src/influence.hpp:
//                     1201-1292: duplicate-point skips, caustic phase, beam
//                     width bound, receiver-range walk); one compact record per
//                     segment that brackets at least one receiver range.
//  influence3d_kernel warp-cooperative evaluation of the (segment, range,
//                     bearing) work of 32 records at a time: a warp prefix sum
//                     flattens it so lanes stay busy; each lane applies the
//                     bearing rejections and walks the receiver depths in the
//                     segment's depth window (src/influence.hpp:1294-1406),
//                     evaluates InfluenceGeoCore (src/influence.hpp:897-1024)
//                     and adds the contribution into the field, laid out as
//                     the reference's [isz][isx][isy][itheta][iz][ir]
//                     (GetFieldAddr, src/common.hpp:393-405).
//  sqrt3d_kernel      ScalePressure's intensity-to-pressure conversion for
//                     incoherent and semi-coherent runs (src/influence.hpp:
//                     1596-1606); coherent 3-D fields are not scaled.
#include <cuda_runtime.h>

#include "bhcb_internal.h"
#include "device_math.cuh"
#include "trace2d.cuh"
#include "influence2d.cuh"
#include "trace3d.cuh"
#include "ray3d.cuh"

namespace bhcb {

namespace {

constexpr int SEG_BLOCK3 = 32;

struct Cursor3 {
    unsigned long long next = 0, end = 0;
};

__device__ __forceinline__ void emit_seg3(const SegRec3 &rec, SegRec3 *segs, unsigned long long cap,
                                          RunCounters *ctr, Cursor3 &cur, bool &overflow)
{
    if(cur.next == cur.end) {
        unsigned long long b = atomicAdd(&ctr->nseg, (unsigned long long)SEG_BLOCK3);
        if(b + SEG_BLOCK3 > cap) {
            overflow = true;
            return;
        }
        cur.next = b;
        cur.end = b + SEG_BLOCK3;
    }
    static_assert(sizeof(SegRec3) % 16 == 0 && sizeof(SegRec3) == 288, "records are written in 16-byte words");
    const uint4 *src = reinterpret_cast<const uint4 *>(&rec);
    uint4 *dst = reinterpret_cast<uint4 *>(segs + cur.next++);
#pragma unroll
    for(int k = 0; k < (int)(sizeof(SegRec3) / 16); ++k) dst[k] = src[k];
}

// the carried part of InfluenceRayInfo for the 3-D Cartesian geometric beams
struct Infl3 {
    double phase, qOld;
    double ratio1, rcp_q0, rcp_qhat0;
    V3 xs;
    int ir;
};

__device__ __forceinline__ double row_len(const M2 &q, int row, double s)
{
    const double a = q.m[0][row] * s, b = q.m[1][row] * s;
    return sqrt(a * a + b * b);
}

// Step_InfluenceGeoCart, 3-D, up to the receiver loop (src/influence.hpp:1201-1292)
__device__ __forceinline__ bool infl_prologue3(const Ray3 &P0, const Ray3 &P1, Infl3 &inf, const Env3Dev &E,
                                               int job, int is, SegRec3 &rec)
{
    const double ax = P0.x.x - inf.xs.x, ay = P0.x.y - inf.xs.y;
    const double bx = P1.x.x - inf.xs.x, by = P1.x.y - inf.xs.y;
    const double rA = sqrt(ax * ax + ay * ay), rB = sqrt(bx * bx + by * by);
    if(fabs(rA - rB) <= 1.0e3 * spacing_d(rA)) return false;   // IsDuplicatePoint(rB, rA)
    if(is == 0) inf.ir = rB > rA ? 0 : E.nrr - 1;
    V3 rayt = sub3(P1.x, P0.x);
    const double rlen = len3(rayt);
    if(rlen <= 1.0e3 * spacing_d(P1.x.x)) return false;
    rayt = v3(rayt.x / rlen, rayt.y / rlen, rayt.z / rlen);
    V3 e1, e2;
    ray_normal(rayt, P1.phi, true, 1.0, e1, e2);
    const double phaseq = m2_det(P0.q);
    if((phaseq <= 0.0 && inf.qOld > 0.0) || (phaseq >= 0.0 && inf.qOld < 0.0)) inf.phase += BHCB_PI / FLTD(2.0);
    inf.qOld = phaseq;
    const double l1 = max(row_len(P0.q, 0, inf.rcp_q0), row_len(P1.q, 0, inf.rcp_q0));
    const double l2 = max(row_len(P0.q, 1, inf.rcp_qhat0), row_len(P1.q, 1, inf.rcp_qhat0));
    const double ldiag = sqrt(l1 * l1 + l2 * l2);

    // receiver-range walk (src/influence.hpp:1294-1297, 1386-1399): the
    // bracketed ranges of one segment are contiguous
    const double *rr = E.rr;
    const double rmin = min(rA, rB), rmax = max(rA, rB);
    int lo = 0x7fffffff, hi = -1;
    for(;;) {
        const double r = rr[inf.ir];
        if(r >= rmin && r < rmax) {
            lo = min(lo, inf.ir);
            hi = max(hi, inf.ir);
        }
        int irTT;
        if(rB > r) {
            if(inf.ir >= E.nrr - 1) break;
            irTT = inf.ir + 1;
            if(rr[irTT] >= rB) break;
        } else {
            if(inf.ir <= 0) break;
            irTT = inf.ir - 1;
            if(rr[irTT] <= rB) break;
        }
        inf.ir = irTT;
    }
    if(hi < 0) return false;
    rec.x0[0] = P0.x.x; rec.x0[1] = P0.x.y; rec.x0[2] = P0.x.z;
    rec.tau0r = P0.taur;
    rec.tau0i = P0.taui;
    rec.dtaur = P1.taur - P0.taur;
    rec.dtaui = P1.taui - P0.taui;
    rec.rayt[0] = rayt.x; rec.rayt[1] = rayt.y; rec.rayt[2] = rayt.z;
    rec.e1[0] = e1.x; rec.e1[1] = e1.y; rec.e1[2] = e1.z;
    rec.e2[0] = e2.x; rec.e2[1] = e2.y; rec.e2[2] = e2.z;
    rec.rlen = rlen;
    rec.q0[0] = P0.q.m[0][0]; rec.q0[1] = P0.q.m[0][1]; rec.q0[2] = P0.q.m[1][0]; rec.q0[3] = P0.q.m[1][1];
    rec.dq[0] = P1.q.m[0][0] - P0.q.m[0][0];
    rec.dq[1] = P1.q.m[0][1] - P0.q.m[0][1];
    rec.dq[2] = P1.q.m[1][0] - P0.q.m[1][0];
    rec.dq[3] = P1.q.m[1][1] - P0.q.m[1][1];
    rec.rcp_q0 = inf.rcp_q0;
    rec.rcp_qhat0 = inf.rcp_qhat0;
    rec.cnst_num = inf.ratio1 * P1.c * P1.Amp;
    rec.phase0 = P0.Phase + inf.phase;
    rec.qold = inf.qOld;
    rec.ldiag = ldiag;
    rec.zlo = min(P0.x.z, P1.x.z);
    rec.zhi = max(P0.x.z, P1.x.z);
    rec.ir_lo = lo;
    rec.ir_hi = hi;
    rec.job = job;
    rec.is = is;
    rec.ntop = P1.ntop;
    rec.nbot = P1.nbot;
    return true;
}

__global__ void __launch_bounds__(64) trace3d_kernel(const GroupDev *__restrict__ groups, int ngroups,
                                                     long long job_end, SegRec3 *segs, unsigned long long cap,
                                                     RunCounters *ctr, unsigned long long *job_counter)
{
    for(;;) {
        const long long job = (long long)atomicAdd(job_counter, 1ull);
        if(job >= job_end) break;
        const GroupDev &G = groups[find_group(groups, ngroups, job)];
        const Env3Dev &E = *G.env3;
        const Job3 J = job_indices3(E, (int)(job - G.job_base));
        if(J.isz >= E.nsz) { run_error(ctr, ERR_RAYINIT); continue; }
        RayState3 st;
        if(!ray_init3d(E, J, st, ctr)) continue;
        Ray3 &p0 = st.p0;
        Ray3 p1, p2;
        const double alpha = st.alpha, c = st.c;
        // ---- Init_Influence (src/influence.hpp:525-644), 3-D Cartesian geometric
        Infl3 inf;
        inf.ratio1 = sqrt(fabs(cos(alpha)));
        inf.ratio1 *= sqrt(E.dalpha * E.dbeta) / c;
        if(E.gaussian) inf.ratio1 /= FLTD(2.0) * BHCB_PI;
        inf.rcp_q0 = E.dalpha / c;
        inf.rcp_qhat0 = fabs(cos(alpha)) * E.dbeta / c;
        inf.phase = 0.0;
        inf.qOld = m2_det(p0.q);
        inf.xs = p0.x;
        inf.ir = bsearch_gt(E.rr, E.nrr, 0.0);

        int small = 0, is = 0;
        bool overflow = false;
        unsigned long long nsteps = 0;
        Cursor3 cur;
        for(;;) {
            if((nsteps & 31) == 0 && __ldcg(&ctr->err_bits) != 0u) break;
            const bool two = ray_update3d(st, p1, p2, small, E, ctr);
            ++nsteps;
            SegRec3 rec;
            if(infl_prologue3(p0, p1, inf, E, (int)job, is, rec)) emit_seg3(rec, segs, cap, ctr, cur, overflow);
            ++is;
            if(two) {
                if(infl_prologue3(p1, p2, inf, E, (int)job, is, rec)) emit_seg3(rec, segs, cap, ctr, cur, overflow);
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
            // ---- RayTerminate (src/trace.hpp:391-477), 3-D
            if(ray_stops3d(st, small, E)) break;
            if(is >= MAXN_STEPS - 3) {
                run_warn(ctr, WARN_ONERAY_OUTOFMEMORY);
                break;
            }
        }
        for(; cur.next < cur.end; ++cur.next) segs[cur.next].job = -1;
        atomicAdd(&ctr->nsteps, nsteps);
    }
}

// Ray trajectories, 3-D (MainRayMode, src/trace.hpp:485-519) of listed rays:
// every ray of a RunType 'R' run, or the rays of eigen hits re-traced up to the
// hit (EigenModePostWorker, src/mode/eigen.cpp:24-45). One ray per thread.
// limits[i] < 0: no limit; else the ray stops two points after step limits[i].
// COUNT: npts[i] = number of points, bounce counts of the last point in
// bnc[2i], bnc[2i + 1]; otherwise the points (x, y, z) go to pts + 3 off[i].
template<bool COUNT>
__global__ void __launch_bounds__(64) ray3d_kernel(const GroupDev *__restrict__ groups, int ngroups,
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
        auto put = [&](int idx, const Ray3 &p) {
            if(!COUNT && idx < cap) {
                double *q = pts + 3 * (base + idx);
                q[0] = p.x.x;
                q[1] = p.x.y;
                q[2] = p.x.z;
            }
        };
        if(J.isz >= E.nsz) {
            run_error(ctr, ERR_RAYINIT);
            if(COUNT) { npts[i] = 0; bnc[2 * i] = bnc[2 * i + 1] = 0; }
            continue;
        }
        RayState3 st;
        int nsteps = -1, last_top = 0, last_bot = 0;
        if(!ray_init3d(E, J, st, ctr)) {
            put(0, st.p0);
            nsteps = 1;
        } else {
            put(0, st.p0);
            const int limit = limits[i];
            int is = 0, small = 0, prev_top = 0, prev_bot = 0;
            Ray3 p1, p2;
            for(;;) {
                if((is & 31) == 0 && __ldcg(&ctr->err_bits) != 0u) {
                    nsteps = is + 1;
                    last_top = st.p0.ntop;
                    last_bot = st.p0.nbot;
                    break;
                }
                const bool two = ray_update3d(st, p1, p2, small, E, ctr);
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
                if(ray_stops3d(st, small, E)) {
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

constexpr int WARPS3 = 4;

// InfluenceGeoCore, 3-D Cartesian (src/influence.hpp:897-1024): beam-window
// test, then amplitude cnst, weight w, phase and complex delay of one receiver
struct Contrib3 {
    double cnst, w, ph, dr, di;
};
__device__ __forceinline__ bool geo_core3(const SegRec3 &R, double s, double n1, double n2, bool gauss, Contrib3 &o)
{
    double q00 = R.q0[0] + s * R.dq[0], q01 = R.q0[1] + s * R.dq[1];
    double q10 = R.q0[2] + s * R.dq[2], q11 = R.q0[3] + s * R.dq[3];
    q00 *= R.rcp_q0;     // row 0 (m[0][0], m[1][0])
    q10 *= R.rcp_q0;
    q01 *= R.rcp_qhat0;  // row 1 (m[0][1], m[1][1])
    q11 *= R.rcp_qhat0;
    const double qF = q00 * q11 - q10 * q01;
    const double l1 = sqrt(q00 * q00 + q10 * q10);
    const double l2 = sqrt(q01 * q01 + q11 * q11);
    if(nearly_zero(l1) || nearly_zero(l2)) return false;
    if(nearly_zero(qF)) return false;
    const double n1p = fabs((-q01 * n2 + q11 * n1) / qF);
    const double n2p = fabs((q00 * n2 - q10 * n1) / qF);
    const double bw = gauss ? 4.0 : 1.0;
    const double dist = gauss ? n1p + n2p : max(n1p, n2p);
    if(dist > bw * 1.0) return false;
    o.dr = R.tau0r + s * R.dtaur;
    o.di = R.tau0i + s * R.dtaui;
    o.cnst = R.cnst_num / sqrt(fabs(qF));
    o.w = gauss ? exp(FLTD(-0.5) * (n1p * n1p + n2p * n2p)) : (FLTD(1.0) - n1p) * (FLTD(1.0) - n2p);
    o.ph = R.phase0;
    if((qF <= 0.0 && R.qold > 0.0) || (qF >= 0.0 && R.qold < 0.0)) o.ph += BHCB_PI / FLTD(2.0);
    return true;
}

// ApplyContribution's TL branch (src/influence.hpp:448-471)
__device__ __forceinline__ float2 tl_field3(const Contrib3 &o, bool gauss, bool coherent, double omega)
{
    if(coherent) {
        const double a = omega * o.dr - o.ph;
        const double m = exp(omega * o.di);
        double sa, ca;
        sincos(-a, &sa, &ca);
        const double cw = o.cnst * o.w;
        return make_float2((float)(cw * (m * ca)), (float)(cw * (m * sa)));
    }
    double v = o.cnst * exp(omega * o.di);
    v = v * v * o.w;
    if(gauss) v *= FLTD(2.0) * BHCB_PI;
    return make_float2((float)v, 0.0f);
}

// The TL contribution of one receiver in the mixed precision (FP32 q, beam
// window, amplitude and weight with the SFU's approximations; the delay's
// phase omega tau is formed and reduced mod 2 pi in FP64, the rest in FP32).
// Same tests and formulas as geo_core3 + tl_field3.
__device__ __forceinline__ bool geo_tl3_mixed(const SegRec3 &R, double s, double n1, double n2, bool gauss,
                                              bool coherent, double omega, float2 &out)
{
    const float sf = (float)s;
    const float rq0 = (float)R.rcp_q0, rq1 = (float)R.rcp_qhat0;
    const float q00 = fmaf(sf, (float)R.dq[0], (float)R.q0[0]) * rq0;
    const float q10 = fmaf(sf, (float)R.dq[2], (float)R.q0[2]) * rq0;
    const float q01 = fmaf(sf, (float)R.dq[1], (float)R.q0[1]) * rq1;
    const float q11 = fmaf(sf, (float)R.dq[3], (float)R.q0[3]) * rq1;
    const float qF = q00 * q11 - q10 * q01;
    const float eps2 = (float)(DBL_EPS * DBL_EPS);
    if(q00 * q00 + q10 * q10 < eps2 || q01 * q01 + q11 * q11 < eps2) return false;
    if(fabsf(qF) < (float)DBL_EPS) return false;
    const float iq = 1.0f / qF;
    const float n1f = (float)n1, n2f = (float)n2;
    const float n1p = fabsf((q11 * n1f - q01 * n2f) * iq);
    const float n2p = fabsf((q00 * n2f - q10 * n1f) * iq);
    const float dist = gauss ? n1p + n2p : fmaxf(n1p, n2p);
    if(dist > (gauss ? 4.0f : 1.0f)) return false;
    const float cnst = (float)R.cnst_num * rsqrtf(fabsf(qF));
    const float w = gauss ? __expf(-0.5f * (n1p * n1p + n2p * n2p)) : (1.0f - n1p) * (1.0f - n2p);
    const float att = __expf((float)(omega * (R.tau0i + s * R.dtaui)));
    if(coherent) {
        float ph = (float)R.phase0;
        if((qF <= 0.0f && R.qold > 0.0) || (qF >= 0.0f && R.qold < 0.0)) ph += (float)(BHCB_PI / 2.0);
        const double a = omega * (R.tau0r + s * R.dtaur);
        const float ar = (float)(a - 6.28318530717958647692 * rint(a * 0.15915494309189533577));
        float sa, ca;
        __sincosf(ph - ar, &sa, &ca);
        const float cw = cnst * w * att;
        out = make_float2(cw * ca, cw * sa);
    } else {
        float v = cnst * att;
        v = v * v * w;
        if(gauss) v *= (float)(2.0 * BHCB_PI);
        out = make_float2(v, 0.0f);
    }
    return true;
}

// first index with (double)rz >= z (n if none)
__device__ __forceinline__ int first_depth_at_or_above(const float *rz, int n, double z)
{
    int lo = 0, hi = n;
    while(lo < hi) {
        const int m = (lo + hi) >> 1;
        if((double)rz[m] < z) lo = m + 1; else hi = m;
    }
    return lo;
}
// last index with (double)rz <= z (-1 if none)
__device__ __forceinline__ int last_depth_at_or_below(const float *rz, int n, double z)
{
    int lo = 0, hi = n;
    while(lo < hi) {
        const int m = (lo + hi) >> 1;
        if((double)rz[m] <= z) lo = m + 1; else hi = m;
    }
    return lo - 1;
}

// A (range, bearing) pair none of whose depths can pass InfluenceGeoCore's
// beam-window test. With A the row-scaled interpolated q (2x2), the accepted
// normal offsets satisfy (n1, n2) = A (+-n1', +-n2'), so their length is at
// most |A|_F |(n1', n2')| <= |A|_F w (w = 4 for Gaussian n1' + n2' <= 4,
// sqrt 2 for hat max(n1', n2') <= 1). That length is at least the distance
// between the receivers' vertical line and the ray line, m' / |t_xy|, and
// |A(s)|_F is convex in s, so its largest value over the depth window is at
// one of the window's two ends. The margin keeps rounding from dropping a
// contribution the per-receiver test would accept.
__device__ __forceinline__ bool pair_outside_beam(const SegRec3 &R, double dxr, double dyr, double mprime,
                                                  double z_lo, double z_hi, bool gauss)
{
    const double th = sqrt(R.rayt[0] * R.rayt[0] + R.rayt[1] * R.rayt[1]);
    if(!(th > 0.0)) return false;
    const double h = dxr * R.rayt[0] + dyr * R.rayt[1];
    double f = 0.0;
#pragma unroll
    for(int e = 0; e < 2; ++e) {
        const double s = (h + ((e ? z_hi : z_lo) - R.x0[2]) * R.rayt[2]) / R.rlen;
        const double a0 = (R.q0[0] + s * R.dq[0]) * R.rcp_q0, a2 = (R.q0[2] + s * R.dq[2]) * R.rcp_q0;
        const double a1 = (R.q0[1] + s * R.dq[1]) * R.rcp_qhat0, a3 = (R.q0[3] + s * R.dq[3]) * R.rcp_qhat0;
        f = max(f, a0 * a0 + a1 * a1 + a2 * a2 + a3 * a3);
    }
    const double w = gauss ? 4.0 : 1.4142135623730951;
    return mprime > th * w * sqrt(f) * (1.0 + 1e-6) + 1e-9;
}

// Work is flattened twice per warp: (segment, range, bearing) pairs over the
// warp's 32 records, then (pair, depth) items over the pairs that survive the
// bearing rejections, so that every lane evaluates receivers.
// MODE: INFL_TL adds the field; INFL_ARR_COUNT counts the arrival candidates;
// INFL_ARR_FILL writes them (AddArr's inputs, src/influence.hpp:444-447) with
// the key (receiver cell, ray, step) that restores the reference's order.
// INFL_EIG_COUNT / INFL_EIG_FILL: the same for eigenray hits (RecordEigenHit,
// src/eigenrays.hpp:24-40), keyed by (trace group, ray, step, position in the
// receiver-range walk, bearing, depth) — the reference's single-threaded order.
// INFL_TL_MIXED: INFL_TL with the receiver's contribution in mixed precision.
enum { INFL_TL = 0, INFL_ARR_COUNT = 1, INFL_ARR_FILL = 2, INFL_EIG_COUNT = 3, INFL_EIG_FILL = 4, INFL_TL_MIXED = 5 };
template<int MODE>
__global__ void __launch_bounds__(32 * WARPS3) influence3d_kernel(
    const SegRec3 *__restrict__ segs, unsigned long long nseg, const GroupDev *__restrict__ groups, int ngroups,
    float2 *field, RunCounters *ctr, ArrCand *cands, uint64_t *keys, uint32_t *vals, unsigned long long cand_cap,
    unsigned long long *cursor, ArrKeyBits kb)
{
    // per record of the warp's chunk
    __shared__ int s_incl[WARPS3][32];
    __shared__ int s_grp[WARPS3][32];
    __shared__ long long s_fbase[WARPS3][32];    // field offset of (isz, isx, isy)
    __shared__ double s_xs[WARPS3][32], s_ys[WARPS3][32];
    // per surviving pair of a 32-pair batch
    __shared__ int s_pincl[WARPS3][32];
    __shared__ int s_prec[WARPS3][32], s_piz0[WARPS3][32], s_pmeta[WARPS3][32];
    __shared__ double s_pdx[WARPS3][32], s_pdy[WARPS3][32];
    __shared__ long long s_poff[WARPS3][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned long long nchunk = (nseg + 31) / 32;
    unsigned long long nevals = 0;
    for(unsigned long long ch = (unsigned long long)blockIdx.x * WARPS3 + w; ch < nchunk;
        ch += (unsigned long long)gridDim.x * WARPS3) {
        const unsigned long long idx = ch * 32 + lane;
        int n = 0, g = 0;
        if(idx < nseg) {
            const int job = __ldg(&segs[idx].job);
            if(job >= 0) {
                g = find_group(groups, ngroups, job);
                const GroupDev &G = groups[g];
                const Env3Dev &E = *G.env3;
                const int lo = __ldg(&segs[idx].ir_lo), hi = __ldg(&segs[idx].ir_hi);
                n = (hi - lo + 1) * E.ntheta;
                const Job3 J = job_indices3(E, (int)(job - G.job_base));
                s_fbase[w][lane] = G.field_base
                    + (long long)(((size_t)J.isz * E.nsx + J.isx) * E.nsy + J.isy) * E.ntheta * E.nrz * E.nrr;
                s_xs[w][lane] = E.sx[J.isx];
                s_ys[w][lane] = E.sy[J.isy];
            }
        }
        int incl = n;
#pragma unroll
        for(int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if(lane >= o) incl += v;
        }
        s_incl[w][lane] = incl;
        s_grp[w][lane] = g;
        __syncwarp();
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        for(int pb = 0; pb < total; pb += 32) {
            // ---- pair stage: bearing rejections and the depth window
            const int k = pb + lane;
            int m = 0;
            if(k < total) {
                int lo = 0, hi = 31;   // first record j with incl[j] > k
                while(lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if(s_incl[w][mid] > k) hi = mid; else lo = mid + 1;
                }
                const int j = lo;
                const int local = k - (j ? s_incl[w][j - 1] : 0);
                const SegRec3 &R = segs[ch * 32 + j];
                const Env3Dev &E = *groups[s_grp[w][j]].env3;
                const int itheta = local % E.ntheta;
                const int ir = R.ir_lo + local / E.ntheta;
                const double xsx = s_xs[w][j], xsy = s_ys[w][j];
                const double tc = E.tcs[2 * itheta], ts = E.tcs[2 * itheta + 1];
                const double rr = E.rr[ir];
                const double xrx = xsx + rr * tc, xry = xsy + rr * ts;
                const double rtx = R.rayt[0], rty = R.rayt[1];
                const double dxr = xrx - R.x0[0], dyr = xry - R.x0[1];
                const bool gauss = E.gaussian != 0;
                const double mprime = fabs(dxr * (-rty) + dyr * rtx);
                bool keep = gauss || !(mprime > 1.0 * R.ldiag);
                keep = keep && !((xrx - xsx) * (R.x0[0] - xsx) + (xry - xsy) * (R.x0[1] - xsy) < 0.0);
                const double nrz = rtx * tc - rty * (-ts);
                keep = keep && !(fabs(nrz) < 1e-9);
                if(keep) {
                    const double Lz = (gauss ? 4.0 : 1.0) * R.ldiag / fabs(nrz);
                    const double zmin = R.zlo - Lz, zmax = R.zhi + Lz;
                    // receiver depths are sorted: the window is the index range [iz0, iz1]
                    const int iz0 = first_depth_at_or_above(E.rz, E.nrz, zmin);
                    const int iz1 = last_depth_at_or_below(E.rz, E.nrz, zmax);
                    if(iz0 <= iz1
                       && !pair_outside_beam(R, dxr, dyr, mprime, (double)E.rz[iz0], (double)E.rz[iz1], gauss)) {
                        m = iz1 - iz0 + 1;
                        s_prec[w][lane] = j;
                        s_piz0[w][lane] = iz0;
                        s_pdx[w][lane] = dxr;
                        s_pdy[w][lane] = dyr;
                        s_poff[w][lane] = s_fbase[w][j] + (long long)itheta * E.nrz * E.nrr + ir;
                        s_pmeta[w][lane] = (itheta << 20) | ir;
                    }
                }
            }
            int pincl = m;
#pragma unroll
            for(int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, pincl, o);
                if(lane >= o) pincl += v;
            }
            s_pincl[w][lane] = pincl;
            __syncwarp();
            const int ptotal = __shfl_sync(0xffffffffu, pincl, 31);
            // ---- receiver stage: one (pair, depth) item per lane
            for(int q = lane; q < ptotal; q += 32) {
                int lo = 0, hi = 31;
                while(lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if(s_pincl[w][mid] > q) hi = mid; else lo = mid + 1;
                }
                const int pi = lo;
                const int iz = s_piz0[w][pi] + q - (pi ? s_pincl[w][pi - 1] : 0);
                const int j = s_prec[w][pi];
                const SegRec3 &R = segs[ch * 32 + j];
                const Env3Dev &E = *groups[s_grp[w][j]].env3;
                const double dxr = s_pdx[w][pi], dyr = s_pdy[w][pi];
                const double dz = (double)E.rz[iz] - R.x0[2];
                const double sv = (dxr * R.rayt[0] + dyr * R.rayt[1] + dz * R.rayt[2]) / R.rlen;
                const double n1 = fabs(dxr * R.e1[0] + dyr * R.e1[1] + dz * R.e1[2]);
                const double n2 = fabs(dxr * R.e2[0] + dyr * R.e2[1] + dz * R.e2[2]);
                if(MODE == INFL_TL_MIXED) {
                    float2 v;
                    if(!geo_tl3_mixed(R, sv, n1, n2, E.gaussian != 0, E.coherent != 0,
                                      FLTD(2.0) * BHCB_PI * E.freq0, v))
                        continue;
                    ++nevals;
                    atomicAdd(field + s_poff[w][pi] + (long long)iz * E.nrr, v);
                    continue;
                }
                Contrib3 o;
                if(!geo_core3(R, sv, n1, n2, E.gaussian != 0, o)) continue;
                ++nevals;
                const long long cell = s_poff[w][pi] + (long long)iz * E.nrr;
                if(MODE == INFL_TL) {
                    const double omega = FLTD(2.0) * BHCB_PI * E.freq0;
                    atomicAdd(field + cell, tl_field3(o, E.gaussian != 0, E.coherent != 0, omega));
                } else if(MODE == INFL_EIG_FILL) {
                    const unsigned long long i = atomicAdd(cursor, 1ull);
                    if(i >= cand_cap) continue;
                    const int itheta = s_pmeta[w][pi] >> 20, ir = s_pmeta[w][pi] & 0xfffff;
                    // the walk visits the bracketed ranges towards rB: ascending when rB > rA
                    const double xsx = s_xs[w][j], xsy = s_ys[w][j];
                    const double ax = R.x0[0] - xsx, ay = R.x0[1] - xsy;
                    const double bx = ax + R.rayt[0] * R.rlen, by = ay + R.rayt[1] * R.rlen;
                    const bool up = bx * bx + by * by > ax * ax + ay * ay;
                    const int walk = up ? ir - R.ir_lo : R.ir_hi - ir;
                    ArrCand c;
                    c.amp = c.phase = c.delay_re = c.delay_im = 0.0;
                    c.rcvr_decl = 0.0f;
                    c.ntop = R.is;
                    c.nbot = ir;
                    c.job = R.job;
                    c.aux = itheta;
                    c.rcvr_azim = __int_as_float(iz);
                    cands[i] = c;
                    keys[i] = ((uint64_t)s_grp[w][j] << kb.sh_cell) | ((uint64_t)R.job << kb.sh_job)
                        | ((uint64_t)R.is << kb.sh_is) | ((uint64_t)walk << kb.sh_walk)
                        | ((uint64_t)itheta << kb.sh_theta) | (uint64_t)iz;
                    vals[i] = (uint32_t)i;
                } else if(MODE == INFL_ARR_FILL) {
                    const unsigned long long i = atomicAdd(cursor, 1ull);
                    if(i >= cand_cap) continue;
                    ArrCand c;
                    c.amp = o.cnst * o.w;
                    c.phase = o.ph;
                    c.delay_re = o.dr;
                    c.delay_im = o.di;
                    // ReceiverAngles, 3-D (src/influence.hpp:123-138)
                    const double rtx = R.rayt[0], rty = R.rayt[1];
                    c.rcvr_decl = (float)((180.0 / BHCB_PI) * atan2(R.rayt[2], sqrt(rtx * rtx + rty * rty)));
                    c.rcvr_azim = (float)((180.0 / BHCB_PI) * atan2(rty, rtx));
                    c.ntop = R.ntop;
                    c.nbot = R.nbot;
                    c.job = R.job;
                    c.aux = 0;
                    cands[i] = c;
                    keys[i] = ((uint64_t)cell << kb.sh_cell) | ((uint64_t)R.job << kb.sh_job) | (uint64_t)R.is;
                    vals[i] = (uint32_t)i;
                }
            }
            __syncwarp();
        }
        __syncwarp();
    }
    // one counter update per warp
#pragma unroll
    for(int o = 16; o > 0; o >>= 1) nevals += __shfl_down_sync(0xffffffffu, nevals, o);
    if(MODE != INFL_ARR_FILL && MODE != INFL_EIG_FILL && lane == 0 && nevals) atomicAdd(&ctr->nevals, nevals);
}

// eigen hits in sorted order (RecordEigenHit layout, include/bhc/structs.hpp:353-361)
__global__ void eigen_emit3_kernel(const uint32_t *__restrict__ vals, const ArrCand *__restrict__ cands,
                                   unsigned long long n, const GroupDev *__restrict__ groups, int ngroups,
                                   EigenHitRec *hits, int32_t *group_of_hit)
{
    for(unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < n;
        k += (unsigned long long)gridDim.x * blockDim.x) {
        const ArrCand &c = cands[vals[k]];
        const int g = find_group(groups, ngroups, c.job);
        const Job3 J = job_indices3(*groups[g].env3, (int)((long long)c.job - groups[g].job_base));
        EigenHitRec h;
        h.is = c.ntop;
        h.itheta = c.aux;
        h.ir = c.nbot;
        h.iz = __float_as_int(c.rcvr_azim);
        h.isx = J.isx;
        h.isy = J.isy;
        h.isz = J.isz;
        h.ialpha = J.ialpha;
        h.ibeta = J.ibeta;
        hits[k] = h;
        group_of_hit[k] = g;
    }
}

__global__ void sqrt3d_kernel(float2 *f, long long n)
{
    for(long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        f[i] = make_float2(sqrtf(f[i].x), 0.0f);
}

} // namespace

cudaError_t launch_rays3d(const GroupDev *groups, int ngroups, const long long *jobs, const int *limits, int nitems,
                          const long long *off, double *pts, int *npts, int *bnc, RunCounters *ctr, bool count,
                          int sm_count, cudaStream_t st)
{
    if(nitems <= 0) return cudaSuccess;
    int grid = (nitems + 63) / 64;
    if(grid > sm_count * 16) grid = sm_count * 16;
    if(count)
        ray3d_kernel<true><<<grid, 64, 0, st>>>(groups, ngroups, jobs, limits, nitems, off, pts, npts, bnc, ctr);
    else
        ray3d_kernel<false><<<grid, 64, 0, st>>>(groups, ngroups, jobs, limits, nitems, off, pts, npts, bnc, ctr);
    return cudaGetLastError();
}

cudaError_t launch_trace3d(const GroupDev *groups, int ngroups, long long job_end, SegRec3 *segs,
                           unsigned long long cap, RunCounters *ctr, unsigned long long *job_counter, int grid,
                           cudaStream_t st)
{
    trace3d_kernel<<<grid, 64, 0, st>>>(groups, ngroups, job_end, segs, cap, ctr, job_counter);
    return cudaGetLastError();
}

cudaError_t launch_influence3d(const SegRec3 *segs, unsigned long long nseg, const GroupDev *groups, int ngroups,
                               float2 *field, RunCounters *ctr, int grid, cudaStream_t st, bool mixed)
{
    if(nseg == 0) return cudaSuccess;
    if(mixed)
        influence3d_kernel<INFL_TL_MIXED><<<grid, 32 * WARPS3, 0, st>>>(segs, nseg, groups, ngroups, field, ctr,
                                                                         nullptr, nullptr, nullptr, 0, nullptr,
                                                                         ArrKeyBits{});
    else
        influence3d_kernel<INFL_TL><<<grid, 32 * WARPS3, 0, st>>>(segs, nseg, groups, ngroups, field, ctr, nullptr,
                                                                   nullptr, nullptr, 0, nullptr, ArrKeyBits{});
    return cudaGetLastError();
}

// arrival candidates of a 3-D run: count = true counts them into ctr->nevals;
// otherwise writes them at cursor (cand_cap slots)
cudaError_t launch_arr_gather3d(const SegRec3 *segs, unsigned long long nseg, const GroupDev *groups, int ngroups,
                                bool count, ArrCand *cands, uint64_t *keys, uint32_t *vals,
                                unsigned long long cand_cap, unsigned long long *cursor, RunCounters *ctr,
                                ArrKeyBits kb, int grid, cudaStream_t st)
{
    if(nseg == 0) return cudaSuccess;
    if(kb.eigen) {
        if(count)
            influence3d_kernel<INFL_EIG_COUNT><<<grid, 32 * WARPS3, 0, st>>>(segs, nseg, groups, ngroups, nullptr,
                                                                             ctr, nullptr, nullptr, nullptr, 0, nullptr,
                                                                             kb);
        else
            influence3d_kernel<INFL_EIG_FILL><<<grid, 32 * WARPS3, 0, st>>>(segs, nseg, groups, ngroups, nullptr,
                                                                            ctr, cands, keys, vals, cand_cap, cursor,
                                                                            kb);
    } else if(count)
        influence3d_kernel<INFL_ARR_COUNT><<<grid, 32 * WARPS3, 0, st>>>(segs, nseg, groups, ngroups, nullptr, ctr,
                                                                         nullptr, nullptr, nullptr, 0, nullptr, kb);
    else
        influence3d_kernel<INFL_ARR_FILL><<<grid, 32 * WARPS3, 0, st>>>(segs, nseg, groups, ngroups, nullptr, ctr,
                                                                        cands, keys, vals, cand_cap, cursor, kb);
    return cudaGetLastError();
}

cudaError_t launch_sqrt3d(float2 *f, long long n, int grid, cudaStream_t st)
{
    if(n <= 0) return cudaSuccess;
    sqrt3d_kernel<<<grid, 256, 0, st>>>(f, n);
    return cudaGetLastError();
}

cudaError_t launch_eigen_emit3(const uint32_t *vals, const ArrCand *cands, unsigned long long n,
                               const GroupDev *groups, int ngroups, EigenHitRec *hits, int32_t *group_of_hit,
                               int sm_count, cudaStream_t st)
{
    if(n == 0) return cudaSuccess;
    long long grid = (long long)((n + 255) / 256);
    if(grid > (long long)sm_count * 32) grid = (long long)sm_count * 32;
    eigen_emit3_kernel<<<(int)grid, 256, 0, st>>>(vals, cands, n, groups, ngroups, hits, group_of_hit);
    return cudaGetLastError();
}

} // namespace bhcb
