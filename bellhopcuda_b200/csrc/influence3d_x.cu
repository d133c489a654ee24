// 3-D (BELLHOP3D) geometric beams in ray-centred coordinates ('g' hat, 'b'
// Gaussian; Step_InfluenceGeoRayCen, 3-D branch, src/influence.hpp:1030-1194),
// TL runs, FP64.
//
//  trace3d_rc_kernel      one ray per thread, the shared 3-D ray driver; per
//                         step the sequential part (caustic phase, duplicate
//                         points, the ray normals of the last valid point) and
//                         one record per segment.
//  influence3d_rc_kernel  one thread per (record, receiver depth, bearing):
//                         the receiver-line intercepts of the planes normal to
//                         the ray at both ends (Compute_RayCenCross /
//                         Compute_M_N_R_IR), the Gaussian radius rejections,
//                         then InfluenceGeoCore at every receiver range
//                         bracketed by the two intercepts, walked from A to B.
#include <cuda_runtime.h>

#include "bhcb_internal.h"
#include "device_math.cuh"
#include "trace2d.cuh"
#include "influence2d.cuh"
#include "trace3d.cuh"
#include "ray3d.cuh"

namespace bhcb {

namespace {

struct Cursor3x {
    unsigned long long next = 0, end = 0;
};

constexpr int SEG_BLOCK3X = 32;

__device__ __forceinline__ void emit_rc3(const XSeg3 &rec, XSeg3 *segs, unsigned long long cap, RunCounters *ctr,
                                         Cursor3x &cur, bool &overflow)
{
    if(cur.next == cur.end) {
        const unsigned long long b = atomicAdd(&ctr->nseg, (unsigned long long)SEG_BLOCK3X);
        if(b + SEG_BLOCK3X > cap) {
            overflow = true;
            return;
        }
        cur.next = b;
        cur.end = b + SEG_BLOCK3X;
    }
    static_assert(sizeof(XSeg3) % 16 == 0, "records are written in 16-byte words");
    const uint4 *src = reinterpret_cast<const uint4 *>(&rec);
    uint4 *dst = reinterpret_cast<uint4 *>(segs + cur.next++);
#pragma unroll
    for(int k = 0; k < (int)(sizeof(XSeg3) / 16); ++k) dst[k] = src[k];
}

// the carried part of InfluenceRayInfo for these beams
struct InflRC3 {
    double phase, qOld, ratio1, rcp_q0, rcp_qhat0;
    V3 rn1, rn2;   // ray normals of the last valid point
};

__device__ __forceinline__ void put3(double *d, V3 v)
{
    d[0] = v.x;
    d[1] = v.y;
    d[2] = v.z;
}

// Step_InfluenceGeoRayCen up to the receiver loops, 3-D
__device__ __forceinline__ bool prologue_rc3(const Ray3 &P0, const Ray3 &P1, InflRC3 &inf, const Env3Dev &E,
                                             const RayState3 &st, int job, int is, XSeg3 &rec)
{
    const double phaseq = m2_det(P0.q);
    if((phaseq <= 0.0 && inf.qOld > 0.0) || (phaseq >= 0.0 && inf.qOld < 0.0)) inf.phase += BHCB_PI / FLTD(2.0);
    inf.qOld = phaseq;
    V3 n1b, n2b;
    ray_normal(P1.t, P1.phi, false, P1.c, n1b, n2b);   // RayNormalRayCen
    // IsDuplicatePoint: a constant 0.1 mm for hat beams, 1000 ulps for Gaussian
    const double d = len3(sub3(P1.x, P0.x));
    const double thr = E.gaussian ? 1.0e3 * spacing_d(P1.x.x) : FLTD(1.0e-4);
    if(d <= thr) {
        inf.rn1 = n1b;
        inf.rn2 = n2b;
        return false;
    }
    put3(rec.x0, P0.x);
    put3(rec.n1a, inf.rn1);
    put3(rec.n2a, inf.rn2);
    put3(rec.ta, scl3(P0.c, P0.t));
    put3(rec.x1, P1.x);
    put3(rec.n1b, n1b);
    put3(rec.n2b, n2b);
    put3(rec.tb, scl3(P1.c, P1.t));
    rec.q0[0] = P0.q.m[0][0]; rec.q0[1] = P0.q.m[0][1]; rec.q0[2] = P0.q.m[1][0]; rec.q0[3] = P0.q.m[1][1];
    rec.dq[0] = P1.q.m[0][0] - P0.q.m[0][0];
    rec.dq[1] = P1.q.m[0][1] - P0.q.m[0][1];
    rec.dq[2] = P1.q.m[1][0] - P0.q.m[1][0];
    rec.dq[3] = P1.q.m[1][1] - P0.q.m[1][1];
    rec.tau0r = P0.taur;
    rec.tau0i = P0.taui;
    rec.dtaur = P1.taur - P0.taur;
    rec.dtaui = P1.taui - P0.taui;
    rec.rcp_q0 = inf.rcp_q0;
    rec.rcp_qhat0 = inf.rcp_qhat0;
    rec.cnst_num = inf.ratio1 * P1.c * P1.Amp;
    rec.phase0 = P0.Phase + inf.phase;
    rec.qold = inf.qOld;
    const double bw = E.gaussian ? 4.0 : 1.0;
    rec.maxr_m = bw * max(fabs(P0.q.m[1][1] * inf.rcp_qhat0), fabs(P1.q.m[1][1] * inf.rcp_qhat0));
    rec.maxr_n = bw * max(fabs(P0.q.m[0][0] * inf.rcp_q0), fabs(P1.q.m[0][0] * inf.rcp_q0));
    rec.xs = st.xs.x;
    rec.ys = st.xs.y;
    rec.job = job;
    rec.is = is;
    rec.ntop = P1.ntop;
    rec.nbot = P1.nbot;
    inf.rn1 = n1b;
    inf.rn2 = n2b;
    return true;
}

__global__ void __launch_bounds__(64) trace3d_rc_kernel(const GroupDev *__restrict__ groups, int ngroups,
                                                        long long job_end, XSeg3 *segs, unsigned long long cap,
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
        // Init_Influence (src/influence.hpp:525-644), 3-D ray-centred geometric
        InflRC3 inf;
        inf.ratio1 = sqrt(fabs(cos(st.alpha))) * (sqrt(E.dalpha * E.dbeta) / st.c);
        if(E.gaussian) inf.ratio1 /= FLTD(2.0) * BHCB_PI;
        inf.rcp_q0 = E.dalpha / st.c;
        inf.rcp_qhat0 = fabs(cos(st.alpha)) * E.dbeta / st.c;
        inf.phase = 0.0;
        inf.qOld = m2_det(p0.q);
        ray_normal(p0.t, p0.phi, false, p0.c, inf.rn1, inf.rn2);
        int small = 0, is = 0;
        bool overflow = false;
        unsigned long long nsteps = 0;
        Cursor3x cur;
        for(;;) {
            if((nsteps & 31) == 0 && __ldcg(&ctr->err_bits) != 0u) break;
            const bool two = ray_update3d(st, p1, p2, small, E, ctr);
            ++nsteps;
            XSeg3 rec;
            if(prologue_rc3(p0, p1, inf, E, st, (int)job, is, rec)) emit_rc3(rec, segs, cap, ctr, cur, overflow);
            ++is;
            if(two) {
                if(prologue_rc3(p1, p2, inf, E, st, (int)job, is, rec)) emit_rc3(rec, segs, cap, ctr, cur, overflow);
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

// RToIR (src/influence.hpp:82-89), 3-D receiver ranges
__device__ __forceinline__ int rtoir3(double r, const Env3Dev &E)
{
    const double dr = E.nrr >= 2 ? E.rr[E.nrr - 1] - E.rr[E.nrr - 2] : 0.0;
    double temp = (r - E.rr[0]) / dr;
    if(fabs(temp - round(temp)) < 1e-6) temp = round(temp);
    if(!(temp > -2147483648.0 && temp < 2147483648.0)) return 0;
    return max(min((int)temp, E.nrr - 1), 0);
}

// Compute_RayCenCross + Compute_M_N_R_IR (src/influence.hpp:155-192): returns
// false when the ray normal is parallel to the receiver bearing's radial
__device__ __forceinline__ bool m_n_r_ir(const double *x, const double *n1, const double *n2, const double *t,
                                         double xs, double ys, double zR, double tcx, double tcy, const Env3Dev &E,
                                         double &m, double &n, double &r, int &ir)
{
    const V3 xt = v3(x[0] - xs, x[1] - ys, x[2] - zR);
    const V3 xe1 = cross3(xt, v3(n1[0], n1[1], n1[2]));
    const V3 xe2 = cross3(xt, v3(n2[0], n2[1], n2[2]));
    const double delta = -(tcx * t[0] + tcy * t[1]);
    if(fabs(delta) < FLTD(1e-3)) return false;
    m = (tcx * xe1.x + tcy * xe1.y) / delta;
    n = -(tcx * xe2.x + tcy * xe2.y) / delta;
    r = -(xt.x * t[0] + xt.y * t[1] + xt.z * t[2]) / delta;
    ir = rtoir3(r, E);
    return true;
}

__global__ void __launch_bounds__(128) influence3d_rc_kernel(const XSeg3 *__restrict__ segs, unsigned long long cap,
                                                             const GroupDev *__restrict__ groups, int ngroups,
                                                             float2 *field, RunCounters *ctr, int nzt)
{
    const unsigned long long nseg = min(__ldcg(&ctr->nseg), cap);
    const unsigned long long nitems = nseg * (unsigned long long)nzt;
    unsigned int evals = 0;
    for(unsigned long long it = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; it < nitems;
        it += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned long long k = it / (unsigned)nzt;
        const int rem = (int)(it - k * (unsigned)nzt);
        const XSeg3 &R = segs[k];
        if(R.job < 0) continue;
        const GroupDev &G = groups[find_group(groups, ngroups, R.job)];
        const Env3Dev &E = *G.env3;
        if(rem >= E.nrz * E.ntheta) continue;
        const int iz = rem / E.ntheta, itheta = rem - iz * E.ntheta;
        const double zR = (double)E.rz[iz];
        const double tcx = E.tcs[2 * itheta], tcy = E.tcs[2 * itheta + 1];
        double mA, nA, rA, mB, nB, rB;
        int irA, irB;
        if(!m_n_r_ir(R.x0, R.n1a, R.n2a, R.ta, R.xs, R.ys, zR, tcx, tcy, E, mA, nA, rA, irA)) continue;
        if(!m_n_r_ir(R.x1, R.n1b, R.n2b, R.tb, R.xs, R.ys, zR, tcx, tcy, E, mB, nB, rB, irB)) continue;
        if(E.gaussian) {
            // possible contribution only if the widest beam reaches the nearest receiver
            if(R.maxr_m <= min(fabs(mA), fabs(mB)) && mA * mB >= 0.0) continue;
            if(R.maxr_n <= min(fabs(nA), fabs(nB)) && nA * nB >= 0.0) continue;
        }
        if(irA == irB) continue;
        const Job3 J = job_indices3(E, (int)(R.job - G.job_base));
        float2 *col = field + G.field_base
            + ((((long long)J.isz * E.nsx + J.isx) * E.nsy + J.isy) * E.ntheta + itheta) * E.nrz * E.nrr
            + (long long)iz * E.nrr;
        const double omega = FLTD(2.0) * BHCB_PI * E.freq0;
        const int up = irB <= irA ? 0 : 1;
        for(int ir = irA + up; ir != irB + up; ir += 2 * up - 1) {
            const double s = (E.rr[ir] - rA) / (rB - rA);
            const double n1 = fabs(nA + s * (nB - nA));
            const double n2 = fabs(mA + s * (mB - mA));
            // InfluenceGeoCore, 3-D ray-centred (src/influence.hpp:897-1024)
            double q00 = R.q0[0] + s * R.dq[0], q01 = R.q0[1] + s * R.dq[1];
            double q10 = R.q0[2] + s * R.dq[2], q11 = R.q0[3] + s * R.dq[3];
            q00 *= R.rcp_q0;
            q10 *= R.rcp_q0;
            q01 *= R.rcp_qhat0;
            q11 *= R.rcp_qhat0;
            const double qF = q00 * q11 - q10 * q01;
            if(nearly_zero(qF)) continue;
            const double n1p = fabs((-q01 * n2 + q11 * n1) / qF);
            const double n2p = fabs((q00 * n2 - q10 * n1) / qF);
            // hat: outside the beam past 1; Gaussian ray-centred: no window
            if(!E.gaussian && max(n1p, n2p) > 1.0) continue;
            const double dr = R.tau0r + s * R.dtaur, di = R.tau0i + s * R.dtaui;
            const double cnst = R.cnst_num / sqrt(fabs(qF));
            const double w = E.gaussian ? exp(FLTD(-0.5) * (n1p * n1p + n2p * n2p))
                                        : (FLTD(1.0) - n1p) * (FLTD(1.0) - n2p);
            double ph = R.phase0;
            if((qF <= 0.0 && R.qold > 0.0) || (qF >= 0.0 && R.qold < 0.0)) ph += BHCB_PI / FLTD(2.0);
            float2 v;
            if(E.coherent) {
                const double a = omega * dr - ph;
                const double mm = exp(omega * di);
                double sa, ca;
                sincos(-a, &sa, &ca);
                const double cw = cnst * w;
                v = make_float2((float)(cw * (mm * ca)), (float)(cw * (mm * sa)));
            } else {
                double vv = cnst * exp(omega * di);
                vv = vv * vv * w;
                if(E.gaussian) vv *= FLTD(2.0) * BHCB_PI;
                v = make_float2((float)vv, 0.0f);
            }
            atomicAdd(col + ir, v);
            ++evals;
        }
    }
    for(int o = 16; o > 0; o >>= 1) evals += __shfl_xor_sync(0xffffffffu, evals, o);
    if((threadIdx.x & 31) == 0 && evals) atomicAdd(&ctr->nevals, (unsigned long long)evals);
}

// Arrival candidates (RunType 'A' / 'a') and eigen hits ('E') of the same
// contributions, one thread per (record, receiver depth, bearing), for the
// shared sort and replay (arrivals.cu): arrivals keyed (receiver cell, ray,
// step) with the receiver angles of the segment's direction (ReceiverAngles,
// src/influence.hpp:123-138, rayt = point1.x - point0.x); eigen hits keyed
// (trace group, ray, step, depth, bearing, walk position from A towards B),
// the reference's loop order within a step (src/influence.hpp:1088-1180).
// COUNT: counts into ctr->nevals; otherwise candidate i at atomicAdd(cursor).
template<bool COUNT>
__global__ void __launch_bounds__(128) arr_gather3d_rc_kernel(const XSeg3 *__restrict__ segs, unsigned long long cap,
                                                              const GroupDev *__restrict__ groups, int ngroups,
                                                              ArrCand *cands, uint64_t *keys, uint32_t *vals,
                                                              unsigned long long cand_cap, unsigned long long *cursor,
                                                              RunCounters *ctr, ArrKeyBits kb, int nzt)
{
    const unsigned long long nseg = min(__ldcg(&ctr->nseg), cap);
    const unsigned long long nitems = nseg * (unsigned long long)nzt;
    unsigned long long count = 0;
    for(unsigned long long it = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; it < nitems;
        it += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned long long k = it / (unsigned)nzt;
        const int rem = (int)(it - k * (unsigned)nzt);
        const XSeg3 &R = segs[k];
        if(R.job < 0) continue;
        const int g = find_group(groups, ngroups, R.job);
        const GroupDev &G = groups[g];
        const Env3Dev &E = *G.env3;
        if(rem >= E.nrz * E.ntheta) continue;
        const int iz = rem / E.ntheta, itheta = rem - iz * E.ntheta;
        const double zR = (double)E.rz[iz];
        const double tcx = E.tcs[2 * itheta], tcy = E.tcs[2 * itheta + 1];
        double mA, nA, rA, mB, nB, rB;
        int irA, irB;
        if(!m_n_r_ir(R.x0, R.n1a, R.n2a, R.ta, R.xs, R.ys, zR, tcx, tcy, E, mA, nA, rA, irA)) continue;
        if(!m_n_r_ir(R.x1, R.n1b, R.n2b, R.tb, R.xs, R.ys, zR, tcx, tcy, E, mB, nB, rB, irB)) continue;
        if(E.gaussian) {
            if(R.maxr_m <= min(fabs(mA), fabs(mB)) && mA * mB >= 0.0) continue;
            if(R.maxr_n <= min(fabs(nA), fabs(nB)) && nA * nB >= 0.0) continue;
        }
        if(irA == irB) continue;
        const int local = (int)(R.job - G.job_base);
        const Job3 J = job_indices3(E, local);
        const long long row = G.field_base
            + ((((long long)J.isz * E.nsx + J.isx) * E.nsy + J.isy) * E.ntheta + itheta) * E.nrz * E.nrr
            + (long long)iz * E.nrr;
        const int up = irB <= irA ? 0 : 1;
        int walk = 0;
        for(int ir = irA + up; ir != irB + up; ir += 2 * up - 1, ++walk) {
            const double s = (E.rr[ir] - rA) / (rB - rA);
            const double n1 = fabs(nA + s * (nB - nA));
            const double n2 = fabs(mA + s * (mB - mA));
            double q00 = R.q0[0] + s * R.dq[0], q01 = R.q0[1] + s * R.dq[1];
            double q10 = R.q0[2] + s * R.dq[2], q11 = R.q0[3] + s * R.dq[3];
            q00 *= R.rcp_q0;
            q10 *= R.rcp_q0;
            q01 *= R.rcp_qhat0;
            q11 *= R.rcp_qhat0;
            const double qF = q00 * q11 - q10 * q01;
            if(nearly_zero(qF)) continue;
            const double n1p = fabs((-q01 * n2 + q11 * n1) / qF);
            const double n2p = fabs((q00 * n2 - q10 * n1) / qF);
            if(!E.gaussian && max(n1p, n2p) > 1.0) continue;
            if(COUNT) {
                ++count;
                continue;
            }
            const unsigned long long i = atomicAdd(cursor, 1ull);
            if(i >= cand_cap) continue;
            ArrCand c;
            uint64_t key;
            if(kb.eigen) {
                c.amp = c.phase = c.delay_re = c.delay_im = 0.0;
                c.rcvr_decl = 0.f;
                c.ntop = R.is;
                c.nbot = ir;
                c.job = R.job;
                c.aux = itheta;
                c.rcvr_azim = __int_as_float(iz);
                key = ((uint64_t)g << kb.sh_cell) | ((uint64_t)local << kb.sh_job) | ((uint64_t)R.is << kb.sh_is)
                      | ((uint64_t)iz << kb.sh_walk) | ((uint64_t)itheta << kb.sh_theta) | (uint64_t)walk;
            } else {
                const double w = E.gaussian ? exp(FLTD(-0.5) * (n1p * n1p + n2p * n2p))
                                            : (FLTD(1.0) - n1p) * (FLTD(1.0) - n2p);
                double ph = R.phase0;
                if((qF <= 0.0 && R.qold > 0.0) || (qF >= 0.0 && R.qold < 0.0)) ph += BHCB_PI / FLTD(2.0);
                const double tx = R.x1[0] - R.x0[0], ty = R.x1[1] - R.x0[1], tz = R.x1[2] - R.x0[2];
                c.amp = R.cnst_num / sqrt(fabs(qF)) * w;
                c.phase = ph;
                c.delay_re = R.tau0r + s * R.dtaur;
                c.delay_im = R.tau0i + s * R.dtaui;
                c.rcvr_decl = (float)((180.0 / BHCB_PI) * atan2(tz, sqrt(tx * tx + ty * ty)));
                c.rcvr_azim = (float)((180.0 / BHCB_PI) * atan2(ty, tx));
                c.ntop = R.ntop;
                c.nbot = R.nbot;
                c.job = R.job;
                c.aux = 0;
                key = ((uint64_t)(row + ir) << kb.sh_cell) | ((uint64_t)local << kb.sh_job) | (uint64_t)R.is;
            }
            cands[i] = c;
            keys[i] = key;
            vals[i] = (uint32_t)i;
        }
    }
    if(COUNT && count) atomicAdd(&ctr->nevals, count);
}

} // namespace

cudaError_t launch_arr_gather3d_rc(const XSeg3 *segs, unsigned long long cap, const GroupDev *groups, int ngroups,
                                   bool count, ArrCand *cands, uint64_t *keys, uint32_t *vals,
                                   unsigned long long cand_cap, unsigned long long *cursor, RunCounters *ctr,
                                   ArrKeyBits kb, int nzt, int grid, cudaStream_t st)
{
    if(nzt < 1) nzt = 1;
    if(count)
        arr_gather3d_rc_kernel<true><<<grid, 128, 0, st>>>(segs, cap, groups, ngroups, cands, keys, vals, cand_cap,
                                                           cursor, ctr, kb, nzt);
    else
        arr_gather3d_rc_kernel<false><<<grid, 128, 0, st>>>(segs, cap, groups, ngroups, cands, keys, vals, cand_cap,
                                                            cursor, ctr, kb, nzt);
    return cudaGetLastError();
}

cudaError_t launch_trace3d_rc(const GroupDev *groups, int ngroups, long long job_end, XSeg3 *segs,
                              unsigned long long cap, RunCounters *ctr, unsigned long long *job_counter, int grid,
                              cudaStream_t st)
{
    trace3d_rc_kernel<<<grid, 64, 0, st>>>(groups, ngroups, job_end, segs, cap, ctr, job_counter);
    return cudaGetLastError();
}

cudaError_t launch_influence3d_rc(const XSeg3 *segs, unsigned long long cap, const GroupDev *groups, int ngroups,
                                  float2 *field, RunCounters *ctr, int nzt, int grid, cudaStream_t st)
{
    if(nzt < 1) nzt = 1;
    influence3d_rc_kernel<<<grid, 128, 0, st>>>(segs, cap, groups, ngroups, field, ctr, nzt);
    return cudaGetLastError();
}

} // namespace bhcb
