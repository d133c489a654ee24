// 2-D field-mode kernels for sm_100a.
//
//  trace_kernel     one ray per thread (persistent, work-queue driven); runs
//                   RayInit / RayUpdate / RayTerminate (src/trace.hpp:76-589)
//                   and the sequential part of Step_InfluenceGeoCart
//                   (src/influence.hpp:1201-1294: duplicate-point skip, caustic
//                   phase, receiver-column walk), then appends one compact
//                   segment record per influence segment.
//  influence_kernel warp-cooperative evaluation of the beam-receiver
//                   contributions of 32 segments at a time (InfluenceGeoCore +
//                   ApplyContribution, src/influence.hpp:423-473,897-1024): a
//                   warp prefix-sum flattens (segment, column, depth) work so
//                   every lane stays busy, contributions are reduced into a
//                   range-major accumulator with 8-byte vector atomics.
//  scale_kernel     ScalePressure (src/influence.hpp:1556-1627) fused with the
//                   transpose of the accumulator into the reference layout
//                   [field][isz][iz][ir] (src/common.hpp:393-405).
#include <cuda_runtime.h>
#include <cooperative_groups.h>
#include <cooperative_groups/scan.h>

#include "bhcb_internal.h"
#include "device_math.cuh"
#include "trace2d.cuh"

namespace cg = cooperative_groups;

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

// Append `emit` segments from the converged lanes of this warp; returns the
// first slot index for this lane (or ~0ull when the buffer is full).
__device__ __forceinline__ unsigned long long warp_append(unsigned long long *counter, int emit)
{
    cg::coalesced_group g = cg::coalesced_threads();
    int incl = cg::inclusive_scan(g, emit);
    unsigned long long base = 0;
    if(g.thread_rank() == g.size() - 1) base = atomicAdd(counter, (unsigned long long)incl);
    base = g.shfl(base, g.size() - 1);
    return base + (unsigned long long)(incl - emit);
}

// Sequential prologue of Step_InfluenceGeoCart (2-D): returns true when the
// segment has receiver columns to evaluate and fills rec.
template<typename R> __device__ __forceinline__ bool infl_prologue(
    const RayPt<R> &p0, const RayPt<R> &p1, InflState &inf, const EnvDev &e, R rcp_q0, R ratio1,
    int job, int is, SegRec<R> &rec)
{
    double rA = inf.x.x, rB = p1.x.x;
    V2<double> d = sub2(p1.x, p0.x);
    double rlen = sqrt(dot2(d, d));
    if(rlen < 1.0e3 * spacing_d(p1.x.x)) return false;   // IsSmallValue: duplicate point
    V2<double> rayt = div2(d, rlen);
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
    rec.x0r = p0.x.x;
    rec.x0z = p0.x.y;
    rec.tau0r = p0.taur;
    rec.dtaur = (R)(p1.taur - p0.taur);
    rec.tau0i = (R)p0.taui;
    rec.dtaui = (R)(p1.taui - p0.taui);
    rec.tx = (R)rayt.x;
    rec.tz = (R)rayt.y;
    rec.rlen = (R)rlen;
    rec.q0 = p0.q.x;
    rec.dq = p1.q.x - p0.q.x;
    rec.rcp_q0 = rcp_q0;
    rec.cnst_num = ratio1 * sqrt(p1.c) * p1.Amp;
    const RayPt<R> &pp = e.gaussian ? p1 : p0;
    rec.phase_a = (R)((double)pp.Phase + inf.phase);
    rec.phase_b = (R)(inf.phase + BHCB_PI / FLTD(2.0));
    rec.sigma_seg = max(fabs(p0.q.x), fabs(p1.q.x)) * rcp_q0 / (R)fabs(rayt.x);
    rec.c0 = p0.c;
    rec.tau1r = (R)p1.taur;
    rec.zlo = (R)min(p0.x.y, p1.x.y);
    rec.zhi = (R)max(p0.x.y, p1.x.y);
    rec.rcvr_decl = (R)((180.0 / BHCB_PI) * atan2(rayt.y, rayt.x));
    rec.ir_lo = min(first, last);
    rec.ir_hi = max(first, last);
    rec.job = job;
    rec.is = is;
    rec.ntop = p1.ntop;
    rec.nbot = p1.nbot;
    return true;
}

template<typename R> __device__ __forceinline__ void emit_seg(
    const SegRec<R> &rec, bool emit, SegRec<R> *segs, unsigned long long cap, RunCounters *ctr,
    bool &overflow)
{
    unsigned long long slot = warp_append(&ctr->nseg, emit ? 1 : 0);
    if(emit) {
        if(slot < cap) {
            segs[slot] = rec;
        } else {
            overflow = true;
        }
    }
}

template<typename R> __global__ void __launch_bounds__(64) trace_kernel(
    const GroupDev *__restrict__ groups, int ngroups, long long njobs, SegRec<R> *segs,
    unsigned long long cap, RunCounters *ctr, unsigned long long *job_counter)
{
    for(;;) {
        long long job = (long long)atomicAdd(job_counter, 1ull);
        if(job >= njobs) break;
        const GroupDev &G = groups[find_group(groups, ngroups, job)];
        const EnvDev &e = *G.env;
        int local = (int)(job - G.job_base);
        int nalpha_eff = e.isingle > 0 ? 1 : e.nalpha;
        int ialpha = e.isingle > 0 ? e.isingle - 1 : local % nalpha_eff;
        int isz = local / nalpha_eff;
        if(isz >= e.nsz) { run_error(ctr, ERR_RAYINIT); continue; }

        // ---- RayInit (src/trace.hpp:76-266)
        SegState iSeg{0, 0};
        double alpha = e.alpha[ialpha];
        double SrcDecl = (180.0 / BHCB_PI) * alpha;
        V2<double> xs = mk2(0.0, (double)e.sz[isz]);
        V2<R> tinit = mk2((R)cos(alpha), (R)sin(alpha));
        SSPOut<R> o;
        eval_ssp(xs, tinit, o, e, iSeg, ctr);
        R c = o.c;
        if(e.coherent && ialpha == 0) {
            double dopt = sqrt((double)c / (FLTD(6.0) * e.freq0 * e.rr[e.nrr - 1]));
            int nopt = 2 + (int)((e.alpha[e.nalpha - 1] - e.alpha[0]) / dopt);
            if(e.nalpha < nopt) run_warn(ctr, WARN_TOO_FEW_BEAMS);
        }
        int ibp = min(bsearch_leq2(e.sbp, e.nsbp, SrcDecl), e.nsbp - 2);
        double s = (SrcDecl - e.sbp[2 * ibp]) / (e.sbp[2 * (ibp + 1)] - e.sbp[2 * ibp]);
        float amp0 = (float)((FLTD(1.0) - s) * e.sbp[2 * ibp + 1] + s * e.sbp[2 * (ibp + 1) + 1]);
        if(e.run0 == 'S') {
            float om = (float)(FLTD(2.0) * BHCB_PI * e.freq0);
            amp0 = (float)(amp0 * ((double)sqrtf(2.0f) * fabs(sin(om / (double)c * xs.y * sin(alpha)))));
        }
        RayPt<R> p0, p1, p2;
        p0.x = xs;
        p0.c = c;
        p0.t = div2(tinit, c);
        p0.taur = 0.0;
        p0.taui = 0.0;
        p0.Amp = (R)amp0;
        p0.Phase = (R)0;
        p0.ntop = p0.nbot = 0;
        p0.p = mk2((R)1, (R)0);
        p0.q = e.q_zero_init ? mk2((R)0, (R)0) : mk2((R)0, (R)1);
        HsDev htop = e.top, hbot = e.bot;
        BdState top, bot;
        top.Iseg = bot.Iseg = 0;
        top.lmin = top.lmax = bot.lmin = bot.lmax = 0.0;
        get_bdry_seg(xs, (double)p0.t.x, top, e.btop, e.ntop, e.top_long, htop, true, true, ctr);
        get_bdry_seg(xs, (double)p0.t.x, bot, e.bbot, e.nbot, e.bot_long, hbot, false, true, ctr);
        double dBegTop, dBegBot, dEndTop, dEndBot;
        distances(xs, top, bot, dBegTop, dBegBot);
        if(dBegTop <= 0.0 || dBegBot <= 0.0) {
            run_warn(ctr, WARN_SOURCE_OUTSIDE_BOUNDARIES);
            continue;
        }
        // ---- Init_Influence (src/influence.hpp:525-644), Cartesian geometric
        R ratio1 = (R)sqrt(fabs(cos(alpha)));
        if(e.line_source) ratio1 = (R)1;
        if(e.gaussian) ratio1 = (R)((double)ratio1 / sqrt(FLTD(2.0) * BHCB_PI));
        R rcp_q0 = (R)(e.dalpha / (double)c);
        InflState inf;
        inf.phase = 0.0;
        inf.qOld = (double)p0.q.x;
        inf.x = p0.x;
        inf.ir = bsearch_gt(e.rr, e.nrr, p0.x.x);
        if(p0.t.x < (R)0 && inf.ir > 0) --inf.ir;

        int small = 0, is = 0;
        bool overflow = false;
        unsigned long long nsteps = 0;
        for(;;) {
            if(__ldcg(&ctr->err_bits) != 0u) break;
            bool tr = false, br = false;
            step2d(p0, p1, top, bot, e, iSeg, small, tr, br, ctr);
            ++nsteps;
            get_bdry_seg(p1.x, (double)p1.t.x, top, e.btop, e.ntop, e.top_long, htop, true, false, ctr);
            get_bdry_seg(p1.x, (double)p1.t.x, bot, e.bbot, e.nbot, e.bot_long, hbot, false, false, ctr);
            distances(p1.x, top, bot, dEndTop, dEndBot);
            bool two = tr || br;
            if(two) {
                const BdryPtDev *bd = tr ? e.btop : e.bbot;
                const BdState &bs = tr ? top : bot;
                const BdryPtDev &b0 = bd[bs.Iseg];
                const BdryPtDev &b1 = bd[bs.Iseg + 1];
                V2<R> nI, tI;
                if(tr ? e.top_curv : e.bot_curv) {
                    double sss = dot2(sub2(p1.x, bs.x), mk2(b0.t[0], b0.t[1])) / b0.Len;
                    nI = mk2((R)((FLTD(1.0) - sss) * b0.Noden[0] + sss * b1.Noden[0]),
                             (R)((FLTD(1.0) - sss) * b0.Noden[1] + sss * b1.Noden[1]));
                    tI = mk2((R)((FLTD(1.0) - sss) * b0.Nodet[0] + sss * b1.Nodet[0]),
                             (R)((FLTD(1.0) - sss) * b0.Nodet[1] + sss * b1.Nodet[1]));
                } else {
                    nI = mk2((R)b0.n[0], (R)b0.n[1]);
                    tI = mk2((R)b0.t[0], (R)b0.t[1]);
                }
                reflect2d(p1, p2, tr ? htop : hbot, tr, tI, nI, (R)b0.kappa, e, iSeg, ctr);
                distances(p2.x, top, bot, dEndTop, dEndBot);
            }
            SegRec<R> rec;
            bool em = infl_prologue(p0, p1, inf, e, rcp_q0, ratio1, (int)job, is, rec);
            emit_seg(rec, em, segs, cap, ctr, overflow);
            ++is;
            if(two) {
                em = infl_prologue(p1, p2, inf, e, rcp_q0, ratio1, (int)job, is, rec);
                emit_seg(rec, em, segs, cap, ctr, overflow);
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
            // ---- RayTerminate (src/trace.hpp:391-477), 2-D
            bool leftbox = fabs(p0.x.x) >= e.box_x || fabs(p0.x.y) >= e.box_y;
            bool escaped = (dBegTop < 0.0 && dEndTop < 0.0) || (dBegBot < 0.0 && dEndBot < 0.0);
            bool lost = (double)p0.Amp < FLTD(0.005);
            if(leftbox || lost || escaped) break;
            if(is >= MAXN_STEPS - 3) {
                run_warn(ctr, WARN_ONERAY_OUTOFMEMORY);
                break;
            }
            dBegTop = dEndTop;
            dBegBot = dEndBot;
        }
        atomicAdd(&ctr->nsteps, nsteps);
    }
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

template<typename R> struct alignas(16) SegShared {
    SegRec<R> rec;
};

// Reduce the phase (double) to [-pi, pi] before the bulk-precision sincos.
__device__ __forceinline__ double reduce_2pi(double a)
{
    const double inv2pi = 0.15915494309189533577, twopi = 6.28318530717958647692;
    return a - twopi * rint(a * inv2pi);
}

constexpr int WARPS_PER_CTA = 4;

template<typename R, bool GAUSS, bool COHERENT> __global__ void __launch_bounds__(32 * WARPS_PER_CTA)
influence_kernel(const SegRec<R> *__restrict__ segs, unsigned long long cap,
                 const GroupDev *__restrict__ groups, int ngroups, const double *__restrict__ freqs,
                 float2 *__restrict__ acc, RunCounters *ctr)
{
    // the trace kernel's append counter may exceed the capacity on overflow
    const unsigned long long nseg = min(__ldcg(&ctr->nseg), cap);
    __shared__ SegRec<R> s_rec[WARPS_PER_CTA][32];
    __shared__ int s_pre[WARPS_PER_CTA][33];
    __shared__ int s_izlo[WARPS_PER_CTA][32];
    __shared__ int s_niz[WARPS_PER_CTA][32];
    __shared__ float s_sig[WARPS_PER_CTA][32];   // sigma lower bound for the frequency (Gaussian)
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned long long nchunks = (nseg + 31) / 32;
    unsigned long long evals = 0;
    for(unsigned long long ch = (unsigned long long)blockIdx.x * WARPS_PER_CTA + w; ch < nchunks;
        ch += (unsigned long long)gridDim.x * WARPS_PER_CTA) {
        unsigned long long si = ch * 32 + lane;
        bool valid = si < nseg;
        // stage this chunk's segment records (coalesced 4-byte words)
        {
            const int words = sizeof(SegRec<R>) / 4;
            const uint32_t *src = reinterpret_cast<const uint32_t *>(segs + ch * 32);
            uint32_t *dst = reinterpret_cast<uint32_t *>(&s_rec[w][0]);
            int nvalid = (int)min(32ull, nseg - ch * 32);
            for(int k = lane; k < nvalid * words; k += 32) dst[k] = __ldcs(src + k);
        }
        __syncwarp();
        const SegRec<R> &my = s_rec[w][lane];
        const GroupDev *G = nullptr;
        const EnvDev *e = nullptr;
        int nfreq = 0;
        if(valid) {
            int job = my.job;
            G = &groups[find_group(groups, ngroups, job)];
            e = G->env;
            nfreq = G->nfreq;
        }
        int maxf = nfreq;
        for(int o = 16; o > 0; o >>= 1) maxf = max(maxf, __shfl_xor_sync(0xffffffffu, maxf, o));
        for(int f = 0; f < maxf; ++f) {
            // ---- per-segment work count for frequency f
            int cnt = 0, izlo = 0, niz = 0;
            float sigfloor = 0.f;
            double freq = 0.0;
            if(valid && f < nfreq) {
                freq = freqs[G->freq_base + f];
                R sig = my.sigma_seg;
                if(GAUSS) {
                    R lam = my.c0 / (R)freq;
                    R fl = min((R)FLTD(0.2) * (R)freq * my.tau1r, (R)BHCB_PI * lam);
                    sigfloor = (float)fl;
                    sig = max(sig, fl);
                }
                double rmax = (GAUSS ? 4.0 : 1.0) * (double)sig;
                int ncol = my.ir_hi - my.ir_lo + 1;
                if(e->irregular) {
                    niz = 1;
                    izlo = 0;
                } else if(fabs((double)my.tx) > FLTD(0.50001)) {
                    double zmin = (double)my.zlo - rmax, zmax = (double)my.zhi + rmax;
                    izlo = lower_f(e->rz, e->nrz, zmin);
                    niz = upper_f(e->rz, e->nrz, zmax) - izlo;
                } else {
                    izlo = 0;
                    niz = e->nrz;
                }
                cnt = niz > 0 ? ncol * niz : 0;
            }
            // warp exclusive scan of counts
            int incl = cnt;
            for(int o = 1; o < 32; o <<= 1) {
                int v = __shfl_up_sync(0xffffffffu, incl, o);
                if(lane >= o) incl += v;
            }
            int total = __shfl_sync(0xffffffffu, incl, 31);
            s_pre[w][lane + 1] = incl;
            if(lane == 0) s_pre[w][0] = 0;
            s_izlo[w][lane] = izlo;
            s_niz[w][lane] = niz;
            s_sig[w][lane] = sigfloor;
            __syncwarp();
            evals += (lane == 0) ? (unsigned long long)total : 0ull;
            for(int ev = lane; ev < total; ev += 32) {
                // owning segment: largest k with s_pre[k] <= ev
                int k = 0;
#pragma unroll
                for(int step = 16; step > 0; step >>= 1)
                    if(s_pre[w][k + step] <= ev) k += step;
                const SegRec<R> &S = s_rec[w][k];
                int j = ev - s_pre[w][k];
                int nz = s_niz[w][k];
                int col = j / nz;
                int izi = j - col * nz;
                int ir = S.ir_lo + col;
                int iz = s_izlo[w][k] + izi;
                const GroupDev &GG = groups[find_group(groups, ngroups, S.job)];
                const EnvDev &E = *GG.env;
                double fq = freqs[GG.freq_base + f];
                double zr = E.irregular ? (double)E.rz[ir] : (double)E.rz[iz];
                R dr = (R)(E.rr[ir] - S.x0r), dz = (R)(zr - S.x0z);
                R s = (dr * S.tx + dz * S.tz) / S.rlen;
                R n1 = fabs(dr * (-S.tz) + dz * S.tx);
                R qF = S.q0 + s * S.dq;
                R sigma = fabs(qF * S.rcp_q0);
                R sig0 = sigma;
                if(GAUSS) sigma = max(sigma, (R)s_sig[w][k]);
                R window = (GAUSS ? (R)4 : (R)1) * sigma;
                if(n1 >= window) continue;   // outside the beam (n > W sigma or n == W sigma)
                double delr = S.tau0r + (double)s * (double)S.dtaur;
                R deli = S.tau0i + s * S.dtaui;
                R cnst = S.cnst_num / sqrt(fabs(qF));
                R wgt;
                if(GAUSS) {
                    R a = n1 / sigma;
                    wgt = exp((R)FLTD(-0.5) * a * a) * (sig0 / sigma);
                } else {
                    wgt = (sigma - n1) / sigma;
                }
                bool caustic = (qF <= (R)0 && S.q0 > (R)0) || (qF >= (R)0 && S.q0 < (R)0);
                R ph = caustic ? S.phase_b : S.phase_a;
                double omega = 2.0 * BHCB_PI * fq;
                float2 v;
                if(COHERENT) {
                    R amp = cnst * wgt * exp((R)omega * deli);
                    double ang = reduce_2pi(omega * delr - (double)ph);
                    R sn, cs;
                    if(sizeof(R) == 4) {
                        float sf, cf;
                        sincosf((float)ang, &sf, &cf);
                        sn = (R)sf; cs = (R)cf;
                    } else {
                        double sd, cd;
                        sincos(ang, &sd, &cd);
                        sn = (R)sd; cs = (R)cd;
                    }
                    v = make_float2((float)(amp * cs), (float)(-amp * sn));
                } else {
                    R vv = cnst * exp((R)omega * deli);
                    vv = vv * vv * wgt;
                    if(GAUSS) vv *= (R)sqrt(FLTD(2.0) * BHCB_PI);
                    v = make_float2((float)vv, 0.f);
                }
                int local = (int)((long long)S.job - GG.job_base);
                int nal = E.isingle > 0 ? 1 : E.nalpha;
                int isz = local / nal;
                size_t addr = (size_t)GG.field_base + (size_t)f * GG.field_stride_f
                    + ((size_t)isz * E.nrr + ir) * E.nrz_per_range + (E.irregular ? 0 : iz);
                atomicAdd(&acc[addr], v);
            }
            __syncwarp();
        }
    }
    if(lane == 0 && evals) atomicAdd(&ctr->nevals, evals);
}

// ScalePressure (src/influence.hpp:1556-1627, 2-D) fused with the transpose
// acc[f][isz][ir][iz] -> out[f][isz][iz][ir].
__global__ void scale_kernel(const float2 *__restrict__ acc, float2 *__restrict__ out,
                             const GroupDev *__restrict__ groups, int ngroups)
{
    __shared__ float2 tile[32][33];
    int g = blockIdx.z;
    const GroupDev &G = groups[g];
    const EnvDev &E = *G.env;
    int nz = E.nrz_per_range, nr = E.nrr;
    int nplanes = G.nfreq * E.nsz;
    int tiles_r = (nr + 31) / 32, tiles_z = (nz + 31) / 32;
    for(int t = blockIdx.x; t < nplanes * tiles_r * tiles_z; t += gridDim.x) {
        int plane = t / (tiles_r * tiles_z);
        int rem = t - plane * tiles_r * tiles_z;
        int tr = rem / tiles_z, tz = rem - tr * tiles_z;
        size_t base = (size_t)G.field_base + (size_t)plane * nr * nz;
        // load: rows ir, contiguous iz
        for(int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
            int ir = tr * 32 + yy, iz = tz * 32 + threadIdx.x;
            if(ir < nr && iz < nz) tile[yy][threadIdx.x] = acc[base + (size_t)ir * nz + iz];
        }
        __syncthreads();
        for(int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
            int iz = tz * 32 + yy, ir = tr * 32 + threadIdx.x;
            if(ir < nr && iz < nz) {
                float2 u = tile[threadIdx.x][yy];
                if(!E.coherent) { u.x = sqrtf(u.x); u.y = 0.f; }
                double cnst = FLTD(-1.0), factor;
                double r = E.rr[ir];
                if(E.line_source) factor = (double)(-4.0f * sqrtf(3.14159265f)) * cnst;
                else if(fabs(r) < DBL_EPS) factor = 0.0;
                else factor = cnst / sqrt(fabs(r));
                float ff = (float)factor;
                out[base + (size_t)iz * nr + ir] = make_float2(u.x * ff, u.y * ff);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- launchers
template<typename R> cudaError_t launch_trace(const GroupDev *groups, int ngroups, long long njobs,
                                              void *segs, unsigned long long cap, RunCounters *ctr,
                                              unsigned long long *job_counter, int grid, int block,
                                              cudaStream_t st)
{
    trace_kernel<R><<<grid, block, 0, st>>>(groups, ngroups, njobs, (SegRec<R> *)segs, cap, ctr,
                                            job_counter);
    return cudaGetLastError();
}

template<typename R> cudaError_t launch_influence(const void *segs, unsigned long long nseg,
                                                  const GroupDev *groups, int ngroups,
                                                  const double *freqs, float2 *acc,
                                                  RunCounters *ctr, bool gauss, bool coherent,
                                                  int grid, cudaStream_t st)
{
    const SegRec<R> *s = (const SegRec<R> *)segs;
    int block = 32 * WARPS_PER_CTA;
    if(gauss && coherent)
        influence_kernel<R, true, true><<<grid, block, 0, st>>>(s, nseg, groups, ngroups, freqs, acc, ctr);
    else if(gauss)
        influence_kernel<R, true, false><<<grid, block, 0, st>>>(s, nseg, groups, ngroups, freqs, acc, ctr);
    else if(coherent)
        influence_kernel<R, false, true><<<grid, block, 0, st>>>(s, nseg, groups, ngroups, freqs, acc, ctr);
    else
        influence_kernel<R, false, false><<<grid, block, 0, st>>>(s, nseg, groups, ngroups, freqs, acc, ctr);
    return cudaGetLastError();
}

cudaError_t launch_scale(const float2 *acc, float2 *out, const GroupDev *groups, int ngroups,
                         int grid_x, cudaStream_t st)
{
    dim3 block(32, 8), grid(grid_x, 1, ngroups);
    scale_kernel<<<grid, block, 0, st>>>(acc, out, groups, ngroups);
    return cudaGetLastError();
}

template cudaError_t launch_trace<float>(const GroupDev *, int, long long, void *, unsigned long long,
                                         RunCounters *, unsigned long long *, int, int, cudaStream_t);
template cudaError_t launch_trace<double>(const GroupDev *, int, long long, void *, unsigned long long,
                                          RunCounters *, unsigned long long *, int, int, cudaStream_t);
template cudaError_t launch_influence<float>(const void *, unsigned long long, const GroupDev *, int,
                                             const double *, float2 *, RunCounters *, bool, bool, int,
                                             cudaStream_t);
template cudaError_t launch_influence<double>(const void *, unsigned long long, const GroupDev *, int,
                                              const double *, float2 *, RunCounters *, bool, bool, int,
                                              cudaStream_t);

size_t seg_record_bytes(bool fp64) { return fp64 ? sizeof(SegRec<double>) : sizeof(SegRec<float>); }

} // namespace bhcb
