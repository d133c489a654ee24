// Device helpers shared by the 2-D field kernels: job -> group lookup, the
// reference's binary searches, the sequential influence prologue of
// Step_InfluenceGeoCart, receiver-depth window search and the per-contribution
// math policies.
#pragma once
#include "bhcb_internal.h"
#include "device_math.cuh"
#include "trace2d.cuh"

namespace bhcb {

__device__ __forceinline__ int find_group(const GroupDev *groups, int ngroups, int64_t job)
{
    int lo = 0, hi = ngroups - 1;
    while(lo < hi) {
        int m = (lo + hi + 1) >> 1;
        if(groups[m].job_base <= job) lo = m; else hi = m - 1;
    }
    return lo;
}

// src/common_run.hpp:61-84 (BinarySearchLEQ) on the pattern table
__device__ __forceinline__ int bsearch_leq2(const double *a, int n, double t)
{
    int lo = 0, hi = n;
    while(lo < hi) {
        int m = (lo + hi) / 2;
        if(a[2 * m] > t) hi = m;
        else if(m >= n - 1) return n - 1;
        else if(a[2 * (m + 1)] > t) return m;
        else lo = m + 1;
    }
    return lo;
}
// src/common_run.hpp:119-138 (BinarySearchGT)
__device__ __forceinline__ int bsearch_gt(const double *a, int n, double t)
{
    int lo = -1, hi = n - 1;
    while(lo < hi) {
        int m = (lo + hi + 1) / 2;
        if(a[m] <= t) lo = m;
        else if(m <= 0) return 0;
        else if(a[m - 1] <= t) return m;
        else hi = m - 1;
    }
    return hi;
}

struct InflState {   // the carried part of InfluenceRayInfo (include/bhc/structs.hpp:462-484)
    double phase, qOld;
    V2<double> x;
    int ir;
};

// Sequential prologue of Step_InfluenceGeoCart (2-D): returns true when the
// segment has receiver columns to evaluate and fills rec.
template<typename R, typename RecR> __device__ __forceinline__ bool infl_prologue(
    const RayPt<R> &p0, const RayPt<R> &p1, InflState &inf, const EnvDev &e, R rcp_q0, R ratio1,
    int job, int is, SegRec<RecR> &rec)
{
    double rA = inf.x.x, rB = p1.x.x;
    V2<double> d = sub2(p1.x, p0.x);
    // IsSmallValue(rlen): duplicate point. rlen = |d| is needed only by
    // segments that reach a receiver column; when |d|^2 exceeds four times the
    // squared threshold, rlen is above the threshold whatever the rounding,
    // and the square root waits until the segment is stored.
    const double dd = dot2(d, d);
    const double small_len = 1.0e3 * spacing_d(p1.x.x);
    double rlen = 0.0;
    const bool long_seg = dd > 4.0 * small_len * small_len;
    if(!long_seg) {
        rlen = sqrt(dd);
        if(rlen < small_len) return false;
    }
    double phaseq = (double)p0.q.x;
    if((phaseq <= 0.0 && inf.qOld > 0.0) || (phaseq >= 0.0 && inf.qOld < 0.0))
        inf.phase += BHCB_PI / FLTD(2.0);
    inf.qOld = phaseq;
    // receiver-column walk (src/influence.hpp:1295-1402 loop control)
    double lo = min(rA, rB), hi = max(rA, rB);
    int first = -1, last = -2;
    int ir = inf.ir;
    const double *rr = e.rr;
    for(int guard = 0; guard <= e.nrr; ++guard) {
        double r = rr[ir];
        if(r >= lo && r < hi) {
            if(first < 0) first = ir;
            last = ir;
        }
        int irTT;
        if(rB > r) {
            if(ir >= e.nrr - 1) break;
            irTT = ir + 1;
            if(rr[irTT] >= rB) break;
        } else {
            if(ir <= 0) break;
            irTT = ir - 1;
            if(rr[irTT] <= rB) break;
        }
        ir = irTT;
    }
    inf.ir = ir;
    inf.x = p1.x;
    if(first < 0) return false;
    if(long_seg) rlen = sqrt(dd);
    const V2<double> rayt = div2(d, rlen);
    rec.x0r = p0.x.x;
    rec.x0z = p0.x.y;
    rec.tau0r = p0.taur;
    rec.dtaur = (RecR)(p1.taur - p0.taur);
    rec.tau0i = (RecR)p0.taui;
    rec.dtaui = (RecR)(p1.taui - p0.taui);
    rec.tx = (RecR)rayt.x;
    rec.tz = (RecR)rayt.y;
    rec.rlen = (RecR)rlen;
    rec.q0 = (RecR)p0.q.x;
    rec.dq = (RecR)(p1.q.x - p0.q.x);
    rec.rcp_q0 = (RecR)rcp_q0;
    rec.cnst_num = (RecR)(ratio1 * sqrt(p1.c) * p1.Amp);
    const RayPt<R> &pp = e.gaussian ? p1 : p0;
    rec.phase_a = (RecR)((double)pp.Phase + inf.phase);
    rec.phase_b = (RecR)(inf.phase + BHCB_PI / FLTD(2.0));
    rec.sigma_seg = (RecR)(max(fabs(p0.q.x), fabs(p1.q.x)) * rcp_q0 / (R)fabs(rayt.x));
    rec.c0 = (RecR)p0.c;
    rec.tau1r = (RecR)p1.taur;
    rec.zlo = (RecR)min(p0.x.y, p1.x.y);
    rec.zhi = (RecR)max(p0.x.y, p1.x.y);
    // receiver declination (ReceiverAngles, src/influence.hpp:123-133): arrivals only
    rec.rcvr_decl = e.arrivals ? (RecR)((180.0 / BHCB_PI) * atan2(rayt.y, rayt.x)) : (RecR)0;
    rec.ir_lo = min(first, last);
    rec.ir_hi = max(first, last);
    rec.job = job;
    rec.is = is;
    rec.ntop = p1.ntop;
    rec.nbot = p1.nbot;
    return true;
}

// first index i in [0,n) with (double)a[i] >= v (a ascending), n if none
__device__ __forceinline__ int lower_f(const float *a, int n, double v)
{
    int lo = 0, hi = n;
    while(lo < hi) {
        int m = (lo + hi) >> 1;
        if((double)a[m] < v) lo = m + 1; else hi = m;
    }
    return lo;
}
// first index i with (double)a[i] > v
__device__ __forceinline__ int upper_f(const float *a, int n, double v)
{
    int lo = 0, hi = n;
    while(lo < hi) {
        int m = (lo + hi) >> 1;
        if((double)a[m] <= v) lo = m + 1; else hi = m;
    }
    return lo;
}

// Reduce an angle to [-pi, pi].
__device__ __forceinline__ double reduce_2pi(double a)
{
    const double inv2pi = 0.15915494309189533577, twopi = 6.28318530717958647692;
    return a - twopi * rint(a * inv2pi);
}
__device__ __forceinline__ float reduce_2pi(float a)
{
    const float inv2pi = 0.159154943f, twopi_hi = 6.28318548f, twopi_lo = -1.7484555e-7f;
    float k = rintf(a * inv2pi);
    return fmaf(-k, twopi_lo, fmaf(-k, twopi_hi, a));
}

// Math used per beam-receiver contribution: IEEE in the FP64 kernel, the SFU
// approximations (after explicit range reduction) in the mixed kernel.
template<typename R> struct EvalMath;
template<> struct EvalMath<double> {
    static __device__ __forceinline__ double div(double a, double b) { return a / b; }
    static __device__ __forceinline__ double exp_(double a) { return exp(a); }
    static __device__ __forceinline__ double rsqrt_(double a) { return 1.0 / sqrt(a); }
    static __device__ __forceinline__ void sincos_(double a, double *s, double *c) { sincos(a, s, c); }
};
template<> struct EvalMath<float> {
    static __device__ __forceinline__ float div(float a, float b) { return __fdividef(a, b); }
    static __device__ __forceinline__ float exp_(float a) { return __expf(a); }
    static __device__ __forceinline__ float rsqrt_(float a) { return rsqrtf(a); }
    static __device__ __forceinline__ void sincos_(float a, float *s, float *c) { __sincosf(a, s, c); }
};

} // namespace bhcb
