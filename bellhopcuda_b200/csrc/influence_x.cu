// 2-D field-mode kernels for the influence types beyond geometric Cartesian
// beams (Step_Influence dispatch, src/influence.hpp:1495-1536):
//
//  trace_x_kernel      one ray per thread, FP64, the shared 2-D ray driver;
//                      per step the sequential part of the kind's influence
//                      function (caustic phase, KMAH index, Cerveny epsilon
//                      and gamma, ray-centred normals, the simple-Gaussian
//                      receiver walk) and one record per segment (ray-centred)
//                      or per bracketed receiver range (Cartesian Cerveny,
//                      simple Gaussian beams).
//  influence_x_kernel  one thread per (record, receiver depth): the receiver
//                      ranges between the segment's two normals at that depth
//                      (ray-centred) or the images of the column (Cerveny
//                      Cartesian), and the contributions, reduced into the
//                      range-major accumulator with 8-byte atomics.
//  scale_x_kernel      ScalePressure (src/influence.hpp:1556-1627, 2-D) with
//                      the Cerveny constant -Dalpha sqrt(f) / c(source), fused
//                      with the transpose into [field][isz][iz][ir].
//
// All math is FP64 as in the reference; the contributions are stored as
// complex<float> like the reference's uAllSources.
#include <cuda_runtime.h>

#include "bhcb_internal.h"
#include "device_math.cuh"
#include "trace2d.cuh"
#include "influence2d.cuh"
#include "ray2d.cuh"

namespace bhcb {

namespace {

typedef Cx<double> cxd;

// RToIR (src/influence.hpp:82-89): index of the receiver range at or before r
// on the (uniformly spaced) receiver line. Out-of-range and NaN values map to
// 0, as the reference's float-to-int conversion does on its CPU build.
__device__ __forceinline__ int rtoir(double r, const EnvDev &e)
{
    double temp = (r - e.rr[0]) / e.delta_r;
    if(fabs(temp - round(temp)) < 1e-6) temp = round(temp);
    if(!(temp > -2147483648.0 && temp < 2147483648.0)) return 0;
    return max(min((int)temp, e.nrr - 1), 0);
}

// Compute_N_R_IR (src/influence.hpp:164-172): normal distance of the receiver
// line at depth zR along the normal through x, its range and index.
__device__ __forceinline__ void n_r_ir(double &n, double &r, int &ir, V2<double> x, V2<double> nrm, double zR,
                                       const EnvDev &e)
{
    n = (zR - x.y) / nrm.y;
    r = x.x + n * nrm.x;
    ir = rtoir(r, e);
}

// RayNormalRayCen, 2-D (src/influence.hpp:142-153)
__device__ __forceinline__ V2<double> raycen_normal(const RayPt<double> &p)
{
    return mk2(p.t.y * p.c, -p.t.x * p.c);
}

__device__ __forceinline__ cxd cexp_(cxd z)
{
    double s, c;
    sincos(z.i, &s, &c);
    const double m = exp(z.r);
    return cx<double>(m * c, m * s);
}

// Hermite (src/influence.hpp:323-340): 1 on [0, x1], cubic taper to 0 at x2
__device__ __forceinline__ double hermite(double x, double x1, double x2)
{
    const double ax = fabs(x);
    if(ax <= x1) return 1.0;
    if(ax >= x2) return 0.0;
    const double u = (ax - x1) / (x2 - x1);
    return (1.0 + 2.0 * u) * (1.0 - u) * (1.0 - u);
}

// BranchCut (src/influence.hpp:345-360): KMAH index update across the branch
// cut of sqrt(q)
__device__ __forceinline__ void branch_cut(cxd q1C, cxd q2C, int &kmah, int beam1)
{
    double q1, q2;
    if(beam1 == 'W') {
        q1 = q1C.r;
        q2 = q2C.r;
    } else {
        if(q2C.r >= 0.0) return;
        q1 = q1C.i;
        q2 = q2C.i;
    }
    if((q1 < 0.0 && q2 >= 0.0) || (q1 > 0.0 && q2 <= 0.0)) kmah = -kmah;
}

// The carried part of InfluenceRayInfo for these kinds
// (include/bhc/structs.hpp:462-484).
struct InflX {
    double phase, qOld;
    V2<double> x, rn;         // ray-centred: last valid point and its ray normal
    bool lastValid;
    int kmah, ir;
    cxd gamma, eps1;          // Cerveny: Cartesian gamma at the last point, epsilon
    double ratio1, rcp_q0, radmax;
};

// PickEpsilon, 2-D Cerveny branch (src/influence.hpp:210-266)
__device__ cxd pick_epsilon(double omega, double c, V2<double> gradc, double angle, double dangle, const EnvDev &e,
                            RunCounters *ctr)
{
    double halfwidth = NAN;
    cxd eps = cx<double>(NAN, NAN);
    bool def_hw = false, def_eps = false;
    switch(e.beam1) {
    case 'F': def_hw = def_eps = true; break;
    case 'M':
        halfwidth = sqrt(FLTD(2.0) * c * FLTD(1000.0) * e.rloop / omega);
        def_eps = true;
        break;
    case 'W': {
        const double cz = gradc.y;
        eps = fabs(cz) < DBL_EPS ? cx<double>(1e10, 0.0)
                                 : cx<double>((-sin(angle) / cos(angle * angle)) * c * c / cz, 0.0);
    } break;
    case 'C': run_warn(ctr, WARN_CERVENY_WIDTH_BUGGY); break;
    default: run_warn(ctr, WARN_INVALID_WIDTH_BUGGY); break;
    }
    if(def_eps) {
        if(def_hw) halfwidth = fabs(dangle) < DBL_EPS ? FLTD(0.0) : FLTD(2.0) / ((omega / c) * dangle);
        eps = cx<double>(0.0, FLTD(0.5) * omega * halfwidth * halfwidth);
    }
    return cscl(e.eps_mult, eps);
}

// Compute_eps_pB_qB (src/influence.hpp:300-312)
__device__ __forceinline__ void eps_pb_qb(cxd &eps, cxd &pB, cxd &qB, const RayPt<double> &p, const InflX &inf,
                                          const EnvDev &e)
{
    eps = e.beam1 == 'C' ? cx<double>(0.0, fabs(p.q.x / p.q.y)) : inf.eps1;
    pB = cx<double>(p.p.x + eps.r * p.p.y, eps.i * p.p.y);
    qB = cx<double>(p.q.x + eps.r * p.q.y, eps.i * p.q.y);
}

// Compute_gamma (src/influence.hpp:270-298)
__device__ cxd compute_gamma(const RayPt<double> &p, cxd pB, cxd qB, const EnvDev &e, SegState &iSeg,
                             RunCounters *ctr)
{
    const V2<double> rayt = scl2(p.c, p.t), rayn = mk2(rayt.y, -rayt.x);
    SSPOut<double> o;
    eval_ssp(p.x, p.t, o, e, iSeg, ctr);
    const double csq = o.c * o.c;
    const double cS = dot2(o.gradc, rayt), cN = dot2(o.gradc, rayn);
    const double Tr = rayt.x, Tz = rayt.y;
    if(cabs_(qB) >= DBL_EPS) {
        const cxd a = cscl(Tr * Tr, cdiv(pB, qB));
        return cscl(FLTD(0.5), cadd(a, cx<double>(FLTD(2.0) * cN / csq * Tz * Tr - cS / csq * (Tz * Tz), 0.0)));
    }
    return cx<double>(0.0, 0.0);
}

// Init_Influence (src/influence.hpp:525-644), 2-D, for the kind
template<int KIND> __device__ void init_x(InflX &inf, const RayState2<double> &st, const EnvDev &e, RunCounters *ctr)
{
    const RayPt<double> &p0 = st.p0;
    const double omega = FLTD(2.0) * BHCB_PI * e.freq0;
    inf.radmax = FLTD(50.0) * p0.c / e.freq0;
    inf.ratio1 = sqrt(fabs(cos(st.alpha)));
    if(e.line_source) inf.ratio1 = 1.0;
    if(KIND == INFL_GEO_RAYCEN && e.gaussian) inf.ratio1 /= sqrt(FLTD(2.0) * BHCB_PI);
    inf.rcp_q0 = e.dalpha / p0.c;
    inf.phase = 0.0;
    inf.qOld = KIND == INFL_SGB ? 1.0 : p0.q.x;
    inf.kmah = 1;
    inf.ir = 0;
    inf.eps1 = cx<double>(0.0, 0.0);
    inf.gamma = cx<double>(0.0, 0.0);
    if(KIND == INFL_CERV_RAYCEN || KIND == INFL_CERV_CART) {
        SegState tmp = st.iSeg;   // the source's gradient, as RayInit returned it
        SSPOut<double> o;
        eval_ssp(p0.x, mk2(cos(st.alpha), sin(st.alpha)), o, e, tmp, ctr);
        inf.eps1 = pick_epsilon(omega, p0.c, o.gradc, st.alpha, e.dalpha, e, ctr);
    }
    if(KIND == INFL_CERV_RAYCEN) {
        inf.rn = mk2(0.0, 1.0);
        inf.x = mk2(0.0, 0.0);
        inf.lastValid = false;
    } else {
        inf.rn = raycen_normal(p0);
        inf.x = p0.x;
        inf.lastValid = fabs(inf.rn.y) >= 1e-6;
    }
    if(KIND == INFL_CERV_CART) {
        cxd eps0, pB0, qB0;
        eps_pb_qb(eps0, pB0, qB0, p0, inf, e);
        SegState tmp = st.iSeg;
        inf.gamma = compute_gamma(p0, pB0, qB0, e, tmp, ctr);
    }
}

__device__ __forceinline__ bool duplicate_x(const RayPt<double> &p0, const RayPt<double> &p1)
{
    return fabs(p1.x.x - p0.x.x) < 1.0e3 * spacing_d(p1.x.x);   // IsDuplicatePoint<false>
}

struct Emitter {
    XSeg *segs;
    unsigned long long cap;
    RunCounters *ctr;
    SlotCursor cur;
    bool overflow;
    __device__ __forceinline__ void put(const XSeg &r) { emit_seg(r, segs, cap, ctr, cur, overflow, nullptr); }
};

__device__ __forceinline__ XSeg blank_rec(int job, int is, const RayPt<double> &p1)
{
    XSeg r;
    r.xa = r.za = r.nxa = r.nza = r.xb = r.zb = r.nxb = r.nzb = 0.0;
    r.tau0r = r.tau0i = r.dtaur = r.dtaui = 0.0;
    r.q0r = r.q0i = r.dqr = r.dqi = r.g0r = r.g0i = r.dgr = r.dgi = r.cr = r.ci = 0.0;
    r.amp = r.ph_a = r.ph_b = r.c0 = r.tau1r = r.rcp_q0 = r.radmax = 0.0;
    r.t1x = r.t1y = r.eps_abs = r.sint = r.sgb_a = r.drab = r.dzab = 0.0;
    r.rcvr_decl = (180.0 / BHCB_PI) * atan2(p1.t.y, p1.t.x);
    r.job = job;
    r.is = is;
    r.ir = 0;
    r.ntop = p1.ntop;
    r.nbot = p1.nbot;
    r.kmah0 = 1;
    r.valid = 1;
    r.pad = 0;
    return r;
}

// The sequential part of the kind's Step_Influence for the segment p0 -> p1
// (step index is); returns false when the influence function ends the ray.
template<int KIND> __device__ bool step_x(const RayPt<double> &p0, const RayPt<double> &p1, InflX &inf,
                                          RayState2<double> &st, const EnvDev &e, int job, int is, Emitter &em,
                                          RunCounters *ctr)
{
    if(KIND == INFL_GEO_RAYCEN) {   // Step_InfluenceGeoRayCen (src/influence.hpp:1030-1194), 2-D
        const double phaseq = p0.q.x;
        if((phaseq <= 0.0 && inf.qOld > 0.0) || (phaseq >= 0.0 && inf.qOld < 0.0)) inf.phase += BHCB_PI / FLTD(2.0);
        inf.qOld = phaseq;
        const V2<double> nB = raycen_normal(p1);
        if(fabs(nB.y) < 1e-10) return true;
        if(!duplicate_x(p0, p1)) {
            XSeg r = blank_rec(job, is, p1);
            r.xa = inf.x.x; r.za = inf.x.y; r.nxa = inf.rn.x; r.nza = inf.rn.y;
            r.valid = inf.lastValid;
            r.xb = p1.x.x; r.zb = p1.x.y; r.nxb = nB.x; r.nzb = nB.y;
            r.tau0r = p0.taur; r.tau0i = p0.taui;
            r.dtaur = p1.taur - p0.taur; r.dtaui = p1.taui - p0.taui;
            r.q0r = p0.q.x; r.dqr = p1.q.x - p0.q.x;
            r.amp = inf.ratio1 * sqrt(p1.c) * p1.Amp;
            r.ph_a = (e.gaussian ? p1.Phase : p0.Phase) + inf.phase;
            r.ph_b = inf.phase + BHCB_PI / FLTD(2.0);
            r.c0 = p0.c; r.tau1r = p1.taur; r.rcp_q0 = inf.rcp_q0;
            em.put(r);
        }
        inf.lastValid = true;
        inf.x = p1.x;
        inf.rn = nB;
        return true;
    } else if(KIND == INFL_CERV_RAYCEN) {   // Step_InfluenceCervenyRayCen (src/influence.hpp:653-754)
        cxd eps0, pB0, qB0, eps1, pB1, qB1;
        eps_pb_qb(eps0, pB0, qB0, p0, inf, e);
        eps_pb_qb(eps1, pB1, qB1, p1, inf, e);
        const cxd gamma0 = cdiv(pB0, qB0), gamma1 = cdiv(pB1, qB1);
        const V2<double> nB = raycen_normal(p1);
        if(fabs(nB.y) < DBL_EPS) return true;
        if(duplicate_x(p0, p1)) {
            inf.lastValid = true;
            inf.x = p1.x;
            inf.rn = nB;
            return true;
        }
        const int old_kmah = inf.kmah;
        branch_cut(qB0, qB1, inf.kmah, e.beam1);
        if(inf.lastValid) {   // the contributions need a previous normal
            XSeg r = blank_rec(job, is, p1);
            r.xa = inf.x.x; r.za = inf.x.y; r.nxa = inf.rn.x; r.nza = inf.rn.y;
            r.xb = p1.x.x; r.zb = p1.x.y; r.nxb = nB.x; r.nzb = nB.y;
            r.tau0r = p0.taur; r.tau0i = p0.taui;
            r.dtaur = p1.taur - p0.taur; r.dtaui = p1.taui - p0.taui;
            r.q0r = qB0.r; r.q0i = qB0.i; r.dqr = qB1.r - qB0.r; r.dqi = qB1.i - qB0.i;
            r.g0r = gamma0.r; r.g0i = gamma0.i; r.dgr = gamma1.r - gamma0.r; r.dgi = gamma1.i - gamma0.i;
            r.amp = inf.ratio1 * p1.Amp;
            r.ph_a = p1.Phase;
            r.c0 = p0.c;
            r.radmax = inf.radmax;
            r.t1x = p1.t.x; r.t1y = p1.t.y;
            r.eps_abs = cabs_(eps1);
            r.kmah0 = old_kmah;
            em.put(r);
        }
        inf.lastValid = true;
        inf.x = p1.x;
        inf.rn = nB;
        return true;
    } else if(KIND == INFL_CERV_CART) {   // Step_InfluenceCervenyCart (src/influence.hpp:759-884)
        cxd eps0, pB0, qB0, eps1, pB1, qB1;
        eps_pb_qb(eps0, pB0, qB0, p0, inf, e);
        eps_pb_qb(eps1, pB1, qB1, p1, inf, e);
        const cxd gamma0 = inf.gamma;
        const cxd gamma1 = compute_gamma(p1, pB1, qB1, e, st.iSeg, ctr);
        inf.gamma = gamma1;
        const int old_kmah = inf.kmah;
        branch_cut(qB0, qB1, inf.kmah, e.beam1);
        if(is == 0) return true;                      // the first pair is skipped
        if(p1.x.x > e.rr[e.nrr - 1]) return false;    // past the last receiver: the ray ends
        const double rA = p0.x.x, rB = p1.x.x;
        if(duplicate_x(p0, p1)) return true;
        const int irA = rtoir(rA, e), irB = rtoir(rB, e);
        if(irA >= irB) return true;
        const double eps0abs = cabs_(eps0);
        for(int ir = irA + 1; ir <= irB; ++ir) {
            const double w = (e.rr[ir] - rA) / (rB - rA);
            const V2<double> x = add2(p0.x, scl2(w, sub2(p1.x, p0.x)));
            const V2<double> rayt = add2(p0.t, scl2(w, sub2(p1.t, p0.t)));
            const double c = p0.c + w * (p1.c - p0.c);
            const cxd q = cadd(qB0, cscl(w, csub(qB1, qB0)));
            const cxd gamma = cadd(gamma0, cscl(w, csub(gamma1, gamma0)));
            if(gamma.i > 0.0) {
                run_warn(ctr, WARN_UNBOUNDED_BEAM);
                continue;
            }
            cxd cnst = cscl(inf.ratio1, csqrt_(rdivc(c * eps0abs, q)));
            int kmah = old_kmah;
            branch_cut(qB0, q, kmah, e.beam1);
            if(kmah < 0) cnst = cx<double>(-cnst.r, -cnst.i);
            XSeg r = blank_rec(job, is, p1);
            r.ir = ir;
            r.xb = x.x; r.zb = x.y; r.t1y = rayt.y;
            r.tau0r = p0.taur + w * (p1.taur - p0.taur);
            r.tau0i = p0.taui + w * (p1.taui - p0.taui);
            r.g0r = gamma.r; r.g0i = gamma.i;
            r.cr = cnst.r; r.ci = cnst.i;
            r.amp = p1.Amp;
            r.ph_a = p1.Phase;
            r.radmax = inf.radmax;
            em.put(r);
        }
        return true;
    } else {   // INFL_SGB: Step_InfluenceSGB (src/influence.hpp:1415-1486)
        const double beta = FLTD(0.98);
        const double a = FLTD(-4.0) * log(beta) / (e.dalpha * e.dalpha);
        const double cn = e.dalpha * sqrt(a / BHCB_PI);
        const double rA = p0.x.x, rB = p1.x.x;
        double q = p0.q.x;
        if((q < 0.0 && inf.qOld >= 0.0) || (q > 0.0 && inf.qOld <= 0.0)) inf.phase += BHCB_PI / FLTD(2.0);
        inf.qOld = q;
        while(fabs(rB - rA) > 1.0e3 * spacing_d(rA) && rB > e.rr[inf.ir]) {
            const double w = (e.rr[inf.ir] - rA) / (rB - rA);
            const V2<double> x = add2(p0.x, scl2(w, sub2(p1.x, p0.x)));
            const V2<double> rayt = add2(p0.t, scl2(w, sub2(p1.t, p0.t)));
            q = p0.q.x + w * (p1.q.x - p0.q.x);
            XSeg r = blank_rec(job, is, p1);
            r.ir = inf.ir;
            r.xb = x.x; r.zb = x.y; r.t1y = rayt.y;
            r.tau0r = p0.taur + w * (p1.taur - p0.taur);
            r.tau0i = p0.taui + w * (p1.taui - p0.taui);
            r.sint = ((double)(is + 1) + w) * e.deltas;
            if((q < 0.0 && inf.qOld >= 0.0) || (q > 0.0 && inf.qOld <= 0.0)) inf.phase += BHCB_PI / FLTD(2.0);
            r.sgb_a = a;
            r.amp = inf.ratio1 * cn * p1.Amp;
            r.ph_a = p1.Phase + inf.phase;
            r.drab = rB - rA;
            r.dzab = p1.x.y - p0.x.y;
            r.radmax = inf.radmax;
            em.put(r);
            inf.qOld = q;
            ++inf.ir;
            if(inf.ir >= e.nrr) return false;
        }
        return true;
    }
}

template<int KIND> __global__ void __launch_bounds__(64) trace_x_kernel(
    const GroupDev *__restrict__ groups, int ngroups, long long njobs, XSeg *segs, unsigned long long cap,
    RunCounters *ctr, unsigned long long *job_counter)
{
    for(;;) {
        const long long job = (long long)atomicAdd(job_counter, 1ull);
        if(job >= njobs) break;
        const GroupDev &G = groups[find_group(groups, ngroups, job)];
        const EnvDev &e = *G.env;
        const int local = (int)(job - G.job_base);
        const int nalpha_eff = e.isingle > 0 ? 1 : e.nalpha;
        const int ialpha = e.isingle > 0 ? e.isingle - 1 : local % nalpha_eff;
        const int isz = local / nalpha_eff;
        if(isz >= e.nsz) { run_error(ctr, ERR_RAYINIT); continue; }
        RayState2<double> st;
        if(!ray_init2d(e, ialpha, isz, st, ctr)) continue;
        InflX inf;
        init_x<KIND>(inf, st, e, ctr);
        Emitter em{segs, cap, ctr, SlotCursor{}, false};
        RayPt<double> &p0 = st.p0;
        RayPt<double> p1, p2;
        double dEndTop, dEndBot;
        int small = 0, is = 0;
        unsigned long long nsteps = 0;
        for(;;) {
            if((nsteps & 31) == 0 && __ldcg(&ctr->err_bits) != 0u) break;
            const bool two = ray_update2d(st, p1, p2, small, dEndTop, dEndBot, e, ctr);
            ++nsteps;
            if(!step_x<KIND>(p0, p1, inf, st, e, (int)job, is, em, ctr)) break;
            ++is;
            if(two) {
                if(!step_x<KIND>(p1, p2, inf, st, e, (int)job, is, em, ctr)) break;
                p0 = p2;
                ++is;
            } else {
                p0 = p1;
            }
            if(em.overflow) break;
            if(ray_stops2d(st, dEndTop, dEndBot, e)) break;
            if(is >= MAXN_STEPS - 3) {
                run_warn(ctr, WARN_ONERAY_OUTOFMEMORY);
                break;
            }
            st.dBegTop = dEndTop;
            st.dBegBot = dEndBot;
        }
        if(em.overflow) {
            atomicMin(&ctr->overflow_job, (unsigned int)job);
            run_error(ctr, ERR_SEG_OVERFLOW);
        }
        close_block(segs, em.cur, (unsigned int *)nullptr);
        atomicAdd(&ctr->nsteps, nsteps);
    }
}

// InfluenceGeoCore + ApplyContribution, 2-D TL (src/influence.hpp:423-473,
// 897-1024) at proportional position s along the segment and normal distance
// n1; returns false when the receiver is outside the beam.
__device__ __forceinline__ bool geo_core(const XSeg &S, double s, double n1, double freq, double omega, bool gauss,
                                         bool coherent, float2 &v)
{
    const double qF = S.q0r + s * S.dqr;
    double sigma = fabs(qF * S.rcp_q0);
    const double sig0 = sigma;
    if(gauss) sigma = max(sigma, min(FLTD(0.2) * freq * S.tau1r, BHCB_PI * (S.c0 / freq)));   // AdjustSigma
    if(n1 >= (gauss ? 4.0 : 1.0) * sigma) return false;
    const double cnst = S.amp / sqrt(fabs(qF));
    const double w = gauss ? exp(FLTD(-0.5) * (n1 / sigma) * (n1 / sigma)) * (sig0 / sigma) : (sigma - n1) / sigma;
    const bool caustic = (qF <= 0.0 && S.q0r > 0.0) || (qF >= 0.0 && S.q0r < 0.0);
    const double ph = caustic ? S.ph_b : S.ph_a;
    const double dr = S.tau0r + s * S.dtaur, di = S.tau0i + s * S.dtaui;
    if(coherent) {
        const cxd z = cexp_(cx<double>(omega * di, -(omega * dr - ph)));
        v = make_float2((float)(cnst * w * z.r), (float)(cnst * w * z.i));
    } else {
        double vv = cnst * exp(omega * di);
        vv = vv * vv * w;
        if(gauss) vv *= sqrt(FLTD(2.0) * BHCB_PI);
        v = make_float2((float)vv, 0.f);
    }
    return true;
}

// InfluenceGeoCore's beam test and the parts ApplyContribution hands to
// AddArr / RecordEigenHit (src/influence.hpp:432-451, 897-1024): amplitude
// cnst w, phase and complex delay; false outside the beam.
__device__ __forceinline__ bool geo_parts(const XSeg &S, double s, double n1, double freq, bool gauss, double &amp,
                                          double &ph, double &dr, double &di)
{
    const double qF = S.q0r + s * S.dqr;
    double sigma = fabs(qF * S.rcp_q0);
    const double sig0 = sigma;
    if(gauss) sigma = max(sigma, min(FLTD(0.2) * freq * S.tau1r, BHCB_PI * (S.c0 / freq)));   // AdjustSigma
    if(n1 >= (gauss ? 4.0 : 1.0) * sigma) return false;
    const double cnst = S.amp / sqrt(fabs(qF));
    const double w = gauss ? exp(FLTD(-0.5) * (n1 / sigma) * (n1 / sigma)) * (sig0 / sigma) : (sigma - n1) / sigma;
    amp = cnst * w;
    const bool caustic = (qF <= 0.0 && S.q0r > 0.0) || (qF >= 0.0 && S.q0r < 0.0);
    ph = caustic ? S.ph_b : S.ph_a;
    dr = S.tau0r + s * S.dtaur;
    di = S.tau0i + s * S.dtaui;
    return true;
}

// FlipBeamForImage / FlipNormalForImage (src/influence.hpp:362-377)
__device__ __forceinline__ V2<double> flip_x(V2<double> x, int image, const EnvDev &e)
{
    if(image == 2) return mk2(x.x, FLTD(2.0) * e.top_depth - x.y);
    if(image == 3) return mk2(x.x, FLTD(2.0) * e.bot_depth - x.y);
    return x;
}
__device__ __forceinline__ V2<double> flip_n(V2<double> n, int image)
{
    return mk2(n.x, n.y * (image == 2 ? -1.0 : 1.0));
}

// One thread per (record, receiver depth). The accumulator is [field][isz][ir][iz].
template<int KIND> __global__ void __launch_bounds__(128) influence_x_kernel(
    const XSeg *__restrict__ segs, unsigned long long cap, const GroupDev *__restrict__ groups, int ngroups,
    const double *__restrict__ freqs, float2 *__restrict__ acc, RunCounters *ctr, int nzmax)
{
    const unsigned long long nseg = min(__ldcg(&ctr->nseg), cap);
    const unsigned long long nitems = nseg * (unsigned long long)nzmax;
    unsigned int evals = 0;
    for(unsigned long long it = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; it < nitems;
        it += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned long long k = it / (unsigned)nzmax;
        const int iz = (int)(it - k * (unsigned)nzmax);
        const XSeg &S = segs[k];
        if(S.job < 0) continue;
        const GroupDev &G = groups[find_group(groups, ngroups, S.job)];
        const EnvDev &e = *G.env;
        if(iz >= e.nrz_per_range) continue;
        const int local = (int)((long long)S.job - G.job_base);
        const int nal = e.isingle > 0 ? 1 : e.nalpha;
        const int isz = local / nal;
        const double freq = freqs[G.freq_base];
        const double omega = FLTD(2.0) * BHCB_PI * freq;
        float2 *col = acc + G.acc_base + (long long)isz * e.nrr * G.acc_nz + iz;
        const double zR = (double)e.rz[iz];
        if(KIND == INFL_GEO_RAYCEN) {
            double nA, rA, nB, rB;
            int irA, irB;
            if(!S.valid) {
                nA = 1e10;
                rA = 1e10;
                irA = 0;
            } else {
                n_r_ir(nA, rA, irA, mk2(S.xa, S.za), mk2(S.nxa, S.nza), zR, e);
            }
            n_r_ir(nB, rB, irB, mk2(S.xb, S.zb), mk2(S.nxb, S.nzb), zR, e);
            if(irA == irB) continue;
            // from A to B, as the reference steps (src/influence.hpp:1171-1180)
            const int up = irB <= irA ? 0 : 1;
            for(int ir = irA + up; ir != irB + up; ir += 2 * up - 1) {
                const double s = (e.rr[ir] - rA) / (rB - rA);
                const double n1 = fabs(nA + s * (nB - nA));
                float2 v;
                if(geo_core(S, s, n1, freq, omega, e.gaussian, e.coherent, v)) {
                    atomicAdd(col + (long long)ir * G.acc_nz, v);
                    ++evals;
                }
            }
        } else if(KIND == INFL_CERV_RAYCEN) {
            const cxd qB0 = cx<double>(S.q0r, S.q0i), dq = cx<double>(S.dqr, S.dqi);
            const cxd g0 = cx<double>(S.g0r, S.g0i), dg = cx<double>(S.dgr, S.dgi);
            const double ibw2 = (double)(e.ibeam_window * e.ibeam_window);
            for(int image = 1; image <= e.nimage; ++image) {
                double nA, rA, nB, rB;
                int ir1, ir2;
                n_r_ir(nB, rB, ir2, flip_x(mk2(S.xb, S.zb), image, e), flip_n(mk2(S.nxb, S.nzb), image), zR, e);
                n_r_ir(nA, rA, ir1, flip_x(mk2(S.xa, S.za), image, e), flip_n(mk2(S.nxa, S.nza), image), zR, e);
                for(int ir = ir1 + 1; ir <= ir2; ++ir) {
                    const double w = (e.rr[ir] - rA) / (rB - rA);
                    const cxd q = cadd(qB0, cscl(w, dq));
                    const cxd gamma = cadd(g0, cscl(w, dg));
                    const double n = nA + w * (nB - nA);
                    const double nSq = n * n;
                    if(gamma.i > 0.0) {
                        run_warn(ctr, WARN_UNBOUNDED_BEAM);
                        continue;
                    }
                    if(!(FLTD(-0.5) * omega * gamma.i * nSq < ibw2)) continue;   // beam window
                    const double c = S.c0;
                    const cxd tau = cx<double>(S.tau0r + w * S.dtaur, S.tau0i + w * S.dtaui);
                    // contri = Ratio1 Amp1 sqrt(c |eps1| / q) exp(-i (omega (tau + gamma n^2 / 2) - Phase1))
                    const cxd arg = cadd(tau, cscl(FLTD(0.5) * nSq, gamma));
                    const cxd ex = cexp_(cx<double>(omega * arg.i, -(omega * arg.r - S.ph_a)));
                    cxd contri = cmul(cscl(S.amp, csqrt_(rdivc(c * S.eps_abs, q))), ex);
                    if(e.component == 'V' || e.component == 'H') {
                        const cxd P_n = cmul(cx<double>(0.0, -omega), cmul(cscl(n, gamma), contri));
                        const cxd P_s = cmul(cx<double>(0.0, -omega / c), contri);
                        if(e.component == 'V')
                            contri = cscl(c, cadd(cscl(S.t1x, P_n), cscl(S.t1y, P_s)));
                        else
                            contri = cscl(c, cadd(cscl(-S.t1y, P_n), cscl(S.t1x, P_s)));
                    }
                    int kmah = S.kmah0;
                    branch_cut(qB0, q, kmah, e.beam1);
                    if(kmah < 0) contri = cx<double>(-contri.r, -contri.i);
                    if(image == 2) contri = cx<double>(-contri.r, -contri.i);
                    if(!e.coherent) contri = cx<double>(contri.r * contri.r + contri.i * contri.i, 0.0);
                    contri = cscl(hermite(n, S.radmax, FLTD(2.0) * S.radmax), contri);
                    atomicAdd(col + (long long)ir * G.acc_nz, make_float2((float)contri.r, (float)contri.i));
                    ++evals;
                }
            }
        } else if(KIND == INFL_CERV_CART) {
            const cxd gamma = cx<double>(S.g0r, S.g0i);
            const double ibw2 = (double)(e.ibeam_window * e.ibeam_window);
            cxd contri = cx<double>(0.0, 0.0);
            for(int image = 1; image <= e.nimage; ++image) {
                double deltaz, polarity;
                if(image == 1) {
                    deltaz = zR - S.zb;
                    polarity = 1.0;
                } else if(image == 2) {
                    deltaz = -zR + FLTD(2.0) * e.top_depth - S.zb;
                    polarity = -1.0;
                } else {
                    deltaz = -zR + FLTD(2.0) * e.bot_depth - S.zb;
                    polarity = 1.0;
                }
                if(omega * gamma.i * deltaz * deltaz < ibw2) {
                    // exp(-i (omega (tau + rayt.y dz + gamma dz^2) - Phase1))
                    const cxd arg = cadd(cx<double>(S.tau0r + S.t1y * deltaz, S.tau0i),
                                         cscl(deltaz * deltaz, gamma));
                    const cxd ex = cexp_(cx<double>(omega * arg.i, -(omega * arg.r - S.ph_a)));
                    const double m = polarity * S.amp * hermite(deltaz, S.radmax, FLTD(2.0) * S.radmax);
                    contri = cadd(contri, cscl(m, ex));
                }
            }
            contri = cmul(cx<double>(S.cr, S.ci), contri);
            if(!e.coherent) contri = cx<double>(contri.r * contri.r + contri.i * contri.i, 0.0);
            atomicAdd(col + (long long)S.ir * G.acc_nz, make_float2((float)contri.r, (float)contri.i));
            ++evals;
        } else {   // INFL_SGB
            const double deltaz = zR - S.zb;
            const double cpa = fabs(deltaz * S.drab) / sqrt(S.drab * S.drab + S.dzab * S.dzab);
            const double ds = sqrt(deltaz * deltaz - cpa * cpa);
            const double sx1 = S.sint + ds;
            const double thet = atan(cpa / sx1);
            const double dr = S.tau0r + S.t1y * deltaz, di = S.tau0i;
            const double cnst = S.amp / sqrt(sx1);
            const double w = exp(-S.sgb_a * thet * thet);
            float2 v;
            if(e.coherent) {
                const cxd z = cexp_(cx<double>(omega * di, -(omega * dr - S.ph_a)));
                v = make_float2((float)(cnst * w * z.r), (float)(cnst * w * z.i));
            } else {
                double vv = cnst * exp(omega * di);
                v = make_float2((float)(vv * vv * w), 0.f);
            }
            atomicAdd(col + (long long)S.ir * G.acc_nz, v);
            ++evals;
        }
    }
    for(int o = 16; o > 0; o >>= 1) evals += __shfl_xor_sync(0xffffffffu, evals, o);
    if((threadIdx.x & 31) == 0 && evals) atomicAdd(&ctr->nevals, (unsigned long long)evals);
}

// Arrival candidates (RunType 'A' / 'a') and eigen hits ('E') of the
// ray-centred geometric ('g', 'b') and simple Gaussian ('S') records, one
// thread per (record, receiver depth), in the form arrivals.cu sorts and
// replays: ArrCand with the key (receiver cell, ray, step) for AddArr, or
// (field, ray, step, walk) for RecordEigenHit, the walk restating the
// reference's loop order within a step: receiver depth, then the ranges from
// A towards B for ray-centred beams (src/influence.hpp:1088-1180); the
// receiver range, then the depth for simple Gaussian beams, which reach only
// depths within RadMax of the ray when the run is not TL (src/influence.hpp:
// 1440-1480). COUNT: only counts (ctr->nevals).
template<int KIND, bool COUNT> __global__ void __launch_bounds__(128) arr_gather_x_kernel(
    const XSeg *__restrict__ segs, unsigned long long cap, const GroupDev *__restrict__ groups, int ngroups,
    const double *__restrict__ freqs, ArrCand *cands, uint64_t *keys, uint32_t *vals, unsigned long long cand_cap,
    unsigned long long *cursor, RunCounters *ctr, ArrKeyBits kb, int nzmax)
{
    const unsigned long long nseg = min(__ldcg(&ctr->nseg), cap);
    const unsigned long long nitems = nseg * (unsigned long long)nzmax;
    unsigned long long count = 0;
    for(unsigned long long it = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; it < nitems;
        it += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned long long k = it / (unsigned)nzmax;
        const int iz = (int)(it - k * (unsigned)nzmax);
        const XSeg &S = segs[k];
        if(S.job < 0) continue;
        const GroupDev &G = groups[find_group(groups, ngroups, S.job)];
        const EnvDev &e = *G.env;
        if(iz >= e.nrz_per_range) continue;
        const int local = (int)((long long)S.job - G.job_base);
        const int nal = e.isingle > 0 ? 1 : e.nalpha;
        const int isz = local / nal;
        const int ialpha = e.isingle > 0 ? e.isingle - 1 : local % nal;
        const double freq = freqs[G.freq_base];
        const double zR = (double)e.rz[iz];
        auto emit = [&](int ir, int hi_walk, int lo_walk, double amp, double ph, double dr, double di) {
            if(COUNT) {
                ++count;
                return;
            }
            const unsigned long long i = atomicAdd(cursor, 1ull);
            if(i >= cand_cap) return;
            ArrCand c;
            uint64_t key;
            if(kb.eigen) {
                key = ((uint64_t)G.field_index << kb.sh_cell) | ((uint64_t)local << kb.sh_job)
                      | ((uint64_t)S.is << kb.sh_is) | ((uint64_t)hi_walk << kb.sh_walk) | (uint64_t)lo_walk;
                c.amp = c.phase = c.delay_re = c.delay_im = 0.0;
                c.rcvr_decl = 0.f;
                c.ntop = S.is;      // eigen: step index
                c.nbot = ir;        // eigen: receiver range index
                c.job = iz | (isz << 20);
            } else {
                const long long cell = G.field_base + ((long long)isz * e.nrz_per_range + iz) * e.nrr + ir;
                key = ((uint64_t)cell << kb.sh_cell) | ((uint64_t)local << kb.sh_job) | (uint64_t)S.is;
                c.amp = amp;
                c.phase = ph;
                c.delay_re = dr;
                c.delay_im = di;
                c.rcvr_decl = (float)S.rcvr_decl;
                c.ntop = S.ntop;
                c.nbot = S.nbot;
                c.job = S.job;
            }
            c.aux = ialpha;
            c.rcvr_azim = 0.f;
            cands[i] = c;
            keys[i] = key;
            vals[i] = (uint32_t)i;
        };
        if(KIND == INFL_GEO_RAYCEN) {
            double nA, rA, nB, rB;
            int irA, irB;
            if(!S.valid) {
                nA = 1e10;
                rA = 1e10;
                irA = 0;
            } else {
                n_r_ir(nA, rA, irA, mk2(S.xa, S.za), mk2(S.nxa, S.nza), zR, e);
            }
            n_r_ir(nB, rB, irB, mk2(S.xb, S.zb), mk2(S.nxb, S.nzb), zR, e);
            if(irA == irB) continue;
            const int up = irB <= irA ? 0 : 1;
            int walk = 0;
            for(int ir = irA + up; ir != irB + up; ir += 2 * up - 1, ++walk) {
                const double s = (e.rr[ir] - rA) / (rB - rA);
                const double n1 = fabs(nA + s * (nB - nA));
                double amp, ph, dr, di;
                if(geo_parts(S, s, n1, freq, e.gaussian, amp, ph, dr, di)) emit(ir, iz, walk, amp, ph, dr, di);
            }
        } else {   // INFL_SGB
            const double deltaz = zR - S.zb;
            if(!(fabs(deltaz) < S.radmax)) continue;
            const double cpa = fabs(deltaz * S.drab) / sqrt(S.drab * S.drab + S.dzab * S.dzab);
            const double ds = sqrt(deltaz * deltaz - cpa * cpa);
            const double sx1 = S.sint + ds;
            const double thet = atan(cpa / sx1);
            const double cnst = S.amp / sqrt(sx1);
            const double w = exp(-S.sgb_a * thet * thet);
            emit(S.ir, S.ir, iz, cnst * w, S.ph_a, S.tau0r + S.t1y * deltaz, S.tau0i);
        }
    }
    if(COUNT && count) atomicAdd(&ctr->nevals, count);
}

// ScalePressure, 2-D (src/influence.hpp:1556-1627, with PostProcessTL's
// source sound speed, src/mode/tl.cpp:106-180) fused with the transpose
// acc[f][isz][ir][iz] -> out[f][isz][iz][ir].
__global__ void scale_x_kernel(const float2 *__restrict__ acc, float2 *__restrict__ out,
                               const GroupDev *__restrict__ groups, const double *__restrict__ freqs,
                               RunCounters *ctr)
{
    __shared__ float2 tile[32][33];
    __shared__ double s_cnst;
    const int g = blockIdx.z;
    const GroupDev &G = groups[g];
    const EnvDev &E = *G.env;
    const int nz = E.nrz_per_range, nr = E.nrr;
    const int nplanes = G.nfreq * E.nsz;
    const int tiles_r = (nr + 31) / 32, tiles_z = (nz + 31) / 32;
    const bool cerveny = E.infl_kind == INFL_CERV_RAYCEN || E.infl_kind == INFL_CERV_CART;
    for(int t = blockIdx.x; t < nplanes * tiles_r * tiles_z; t += gridDim.x) {
        const int plane = t / (tiles_r * tiles_z);
        const int rem = t - plane * tiles_r * tiles_z;
        const int tr = rem / tiles_z, tz = rem - tr * tiles_z;
        if(threadIdx.x == 0 && threadIdx.y == 0) {
            double cnst = FLTD(-1.0);
            if(cerveny) {   // -Dalpha sqrt(f) / c at the source, launched horizontally
                const int f = plane / E.nsz, isz = plane - f * E.nsz;
                SegState seg{0, 0};
                SSPOut<double> o;
                eval_ssp(mk2(0.0, (double)E.sz[isz]), mk2(1.0, 0.0), o, E, seg, ctr);
                cnst = -E.dalpha * sqrt(freqs[G.freq_base + f]) / o.c;
            }
            s_cnst = cnst;
        }
        const size_t base = (size_t)G.field_base + (size_t)plane * nr * nz;
        const size_t abase = (size_t)G.acc_base + (size_t)plane * nr * G.acc_nz;
        for(int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
            const int ir = tr * 32 + yy, iz = tz * 32 + threadIdx.x;
            if(ir < nr && iz < nz) tile[yy][threadIdx.x] = acc[abase + (size_t)ir * G.acc_nz + iz];
        }
        __syncthreads();
        const double cnst = s_cnst;
        for(int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
            const int iz = tz * 32 + yy, ir = tr * 32 + threadIdx.x;
            if(ir < nr && iz < nz) {
                float2 u = tile[threadIdx.x][yy];
                if(!E.coherent) { u.x = sqrtf(u.x); u.y = 0.f; }
                double factor;
                const double r = E.rr[ir];
                if(E.line_source) factor = (double)(-4.0f * sqrtf(3.14159265f)) * cnst;
                else if(fabs(r) < DBL_EPS) factor = 0.0;
                else factor = cnst / sqrt(fabs(r));
                const float ff = (float)factor;
                out[base + (size_t)iz * nr + ir] = make_float2(u.x * ff, u.y * ff);
            }
        }
        __syncthreads();
    }
}

} // namespace

cudaError_t launch_trace_x(const GroupDev *groups, int ngroups, long long njobs, XSeg *segs, unsigned long long cap,
                           RunCounters *ctr, unsigned long long *job_counter, int kind, int grid, int block,
                           cudaStream_t st)
{
    switch(kind) {
    case INFL_GEO_RAYCEN:
        trace_x_kernel<INFL_GEO_RAYCEN><<<grid, block, 0, st>>>(groups, ngroups, njobs, segs, cap, ctr, job_counter);
        break;
    case INFL_CERV_RAYCEN:
        trace_x_kernel<INFL_CERV_RAYCEN><<<grid, block, 0, st>>>(groups, ngroups, njobs, segs, cap, ctr, job_counter);
        break;
    case INFL_CERV_CART:
        trace_x_kernel<INFL_CERV_CART><<<grid, block, 0, st>>>(groups, ngroups, njobs, segs, cap, ctr, job_counter);
        break;
    case INFL_SGB:
        trace_x_kernel<INFL_SGB><<<grid, block, 0, st>>>(groups, ngroups, njobs, segs, cap, ctr, job_counter);
        break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_influence_x(const XSeg *segs, unsigned long long cap, const GroupDev *groups, int ngroups,
                               const double *freqs, float2 *acc, RunCounters *ctr, int kind, int nzmax, int grid,
                               cudaStream_t st)
{
    if(nzmax < 1) nzmax = 1;
    switch(kind) {
    case INFL_GEO_RAYCEN:
        influence_x_kernel<INFL_GEO_RAYCEN><<<grid, 128, 0, st>>>(segs, cap, groups, ngroups, freqs, acc, ctr, nzmax);
        break;
    case INFL_CERV_RAYCEN:
        influence_x_kernel<INFL_CERV_RAYCEN><<<grid, 128, 0, st>>>(segs, cap, groups, ngroups, freqs, acc, ctr, nzmax);
        break;
    case INFL_CERV_CART:
        influence_x_kernel<INFL_CERV_CART><<<grid, 128, 0, st>>>(segs, cap, groups, ngroups, freqs, acc, ctr, nzmax);
        break;
    case INFL_SGB:
        influence_x_kernel<INFL_SGB><<<grid, 128, 0, st>>>(segs, cap, groups, ngroups, freqs, acc, ctr, nzmax);
        break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_arr_gather_x(const XSeg *segs, unsigned long long cap, const GroupDev *groups, int ngroups,
                                const double *freqs, int kind, bool count, ArrCand *cands, uint64_t *keys,
                                uint32_t *vals, unsigned long long cand_cap, unsigned long long *cursor,
                                RunCounters *ctr, ArrKeyBits kb, int nzmax, int grid, cudaStream_t st)
{
    if(nzmax < 1) nzmax = 1;
    if(kind == INFL_GEO_RAYCEN) {
        if(count)
            arr_gather_x_kernel<INFL_GEO_RAYCEN, true><<<grid, 128, 0, st>>>(segs, cap, groups, ngroups, freqs, cands,
                                                                             keys, vals, cand_cap, cursor, ctr, kb,
                                                                             nzmax);
        else
            arr_gather_x_kernel<INFL_GEO_RAYCEN, false><<<grid, 128, 0, st>>>(segs, cap, groups, ngroups, freqs,
                                                                              cands, keys, vals, cand_cap, cursor,
                                                                              ctr, kb, nzmax);
    } else if(kind == INFL_SGB) {
        if(count)
            arr_gather_x_kernel<INFL_SGB, true><<<grid, 128, 0, st>>>(segs, cap, groups, ngroups, freqs, cands, keys,
                                                                      vals, cand_cap, cursor, ctr, kb, nzmax);
        else
            arr_gather_x_kernel<INFL_SGB, false><<<grid, 128, 0, st>>>(segs, cap, groups, ngroups, freqs, cands,
                                                                       keys, vals, cand_cap, cursor, ctr, kb, nzmax);
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_scale_x(const float2 *acc, float2 *out, const GroupDev *groups, int ngroups, const double *freqs,
                           RunCounters *ctr, int grid_x, cudaStream_t st)
{
    dim3 block(32, 8), grid(grid_x, 1, ngroups);
    scale_x_kernel<<<grid, block, 0, st>>>(acc, out, groups, freqs, ctr);
    return cudaGetLastError();
}

} // namespace bhcb
