// 2-D field-mode kernels for sm_100a.
//
//  trace_kernel     one ray per thread (persistent, work-queue driven), FP64
//                   ray state, FP32 or FP64 segment records; runs
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

#include "bhcb_internal.h"
#include "device_math.cuh"
#include "trace2d.cuh"
#include "influence2d.cuh"
#include "ray2d.cuh"
#include "tabstage.cuh"

namespace bhcb {

// R: ray state; RecR: segment record (float for the mixed kernel's FP32 influence).
// lanes: rays per warp (16 or 32); the other lanes only help stage the tables.
template<typename R, typename RecR> __global__ void __launch_bounds__(64) trace_kernel(
    const GroupDev *__restrict__ groups, int ngroups, long long njobs, SegRec<RecR> *segs,
    unsigned long long cap, RunCounters *ctr, unsigned long long *job_counter, unsigned int *blk_state,
    unsigned int stage_budget, int lanes)
{
    // tables of the group this CTA's first rays belong to, staged in shared memory
    extern __shared__ __align__(16) unsigned char s_tab[];
    __shared__ EnvDev s_env;
    __shared__ __align__(8) uint64_t s_bar;
    const long long hint = min(njobs - 1, groups[0].job_base + (long long)blockIdx.x * blockDim.x);
    const int gs = find_group(groups, ngroups, hint);
    const bool staged = stage_budget > 0 && stage_env_tables(groups[gs].env, s_env, s_tab, stage_budget, &s_bar, ctr);
    for(;;) {
        // a warp with fewer rays takes fewer divergent paths per step
        if((int)(threadIdx.x & 31) >= lanes) break;
        long long job = (long long)atomicAdd(job_counter, 1ull);
        if(job >= njobs) break;
        const int gi = find_group(groups, ngroups, job);
        const GroupDev &G = groups[gi];
        const EnvDev &e = (staged && gi == gs) ? s_env : *G.env;
        int local = (int)(job - G.job_base);
        int nalpha_eff = e.isingle > 0 ? 1 : e.nalpha;
        int ialpha = e.isingle > 0 ? e.isingle - 1 : local % nalpha_eff;
        int isz = local / nalpha_eff;
        if(isz >= e.nsz) { run_error(ctr, ERR_RAYINIT); continue; }

        // ---- RayInit (src/trace.hpp:76-266)
        RayState2<R> st;
        if(!ray_init2d(e, ialpha, isz, st, ctr)) continue;
        RayPt<R> &p0 = st.p0;
        RayPt<R> p1, p2;
        const double alpha = st.alpha;
        const R c = st.c;
        double dEndTop, dEndBot;
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
        SlotCursor cur;
        for(;;) {
            // another ray's error stops the run (src/trace.hpp:559); polled every 32 steps
            if((nsteps & 31) == 0 && __ldcg(&ctr->err_bits) != 0u) break;
            const bool two = ray_update2d(st, p1, p2, small, dEndTop, dEndBot, e, ctr);
            ++nsteps;
            SegRec<RecR> rec;
            if(infl_prologue(p0, p1, inf, e, rcp_q0, ratio1, (int)job, is, rec))
                emit_seg(rec, segs, cap, ctr, cur, overflow, blk_state);
            ++is;
            if(two) {
                if(infl_prologue(p1, p2, inf, e, rcp_q0, ratio1, (int)job, is, rec))
                    emit_seg(rec, segs, cap, ctr, cur, overflow, blk_state);
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
            if(ray_stops2d(st, dEndTop, dEndBot, e)) break;
            if(is >= MAXN_STEPS - 3) {
                run_warn(ctr, WARN_ONERAY_OUTOFMEMORY);
                break;
            }
            st.dBegTop = dEndTop;
            st.dBegBot = dEndBot;
        }
        close_block(segs, cur, blk_state);
        atomicAdd(&ctr->nsteps, nsteps);
    }
    if(stage_budget > 0 && !staged) stage_drain(&s_bar);
}

// Ray trajectories (MainRayMode, src/trace.hpp:485-519) of listed rays: every
// ray of a RunType 'R' run, or the rays of eigen hits re-traced up to the hit
// (EigenModePostWorker, src/mode/eigen.cpp:24-45). One ray per thread, FP64.
// limits[i] < 0: no limit; else the ray stops two points after step limits[i].
// COUNT: npts[i] = number of points, bounce counts of the last point in
// bnc[2i], bnc[2i + 1]; otherwise the points (r, z) go to pts + off[i].
template<bool COUNT>
__global__ void __launch_bounds__(64) ray_kernel(const GroupDev *__restrict__ groups, int ngroups,
                                                 const long long *__restrict__ jobs, const int *__restrict__ limits,
                                                 int nitems, const long long *__restrict__ off, double2 *pts,
                                                 int *npts, int *bnc, RunCounters *ctr)
{
    for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < nitems; i += gridDim.x * blockDim.x) {
        const long long job = jobs[i];
        const GroupDev &G = groups[find_group(groups, ngroups, job)];
        const EnvDev &e = *G.env;
        const int local = (int)(job - G.job_base);
        const int nalpha_eff = e.isingle > 0 ? 1 : e.nalpha;
        const int ialpha = e.isingle > 0 ? e.isingle - 1 : local % nalpha_eff;
        const int isz = local / nalpha_eff;
        const int cap = COUNT ? 0x7fffffff : npts[i];   // points the count pass found
        const long long base = COUNT ? 0 : off[i];
        auto put = [&](int idx, const RayPt<double> &p) {
            if(!COUNT && idx < cap) pts[base + idx] = make_double2(p.x.x, p.x.y);
        };
        if(isz >= e.nsz) {
            run_error(ctr, ERR_RAYINIT);
            if(COUNT) { npts[i] = 0; bnc[2 * i] = bnc[2 * i + 1] = 0; }
            continue;
        }
        RayState2<double> st;
        int nsteps = -1;
        int last_top = 0, last_bot = 0;
        if(!ray_init2d(e, ialpha, isz, st, ctr)) {
            put(0, st.p0);
            nsteps = 1;
        } else {
            put(0, st.p0);
            const int limit = limits[i];
            int is = 0, small = 0;
            int prev_top = 0, prev_bot = 0;   // bounces of the point before st.p0
            RayPt<double> p1, p2;
            double dEndTop, dEndBot;
            for(;;) {
                if((is & 31) == 0 && __ldcg(&ctr->err_bits) != 0u) {
                    nsteps = is + 1;
                    last_top = st.p0.ntop;
                    last_bot = st.p0.nbot;
                    break;
                }
                const bool two = ray_update2d(st, p1, p2, small, dEndTop, dEndBot, e, ctr);
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
                if(ray_stops2d(st, dEndTop, dEndBot, e)) {
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
                st.dBegTop = dEndTop;
                st.dBegBot = dEndBot;
            }
        }
        if(COUNT) {
            npts[i] = nsteps;
            bnc[2 * i] = last_top;
            bnc[2 * i + 1] = last_bot;
        }
    }
}

constexpr int WARPS_PER_CTA = 4;

// Per (segment, frequency) values computed once by the segment's owner lane.
template<typename R> struct SegFreq {
    R sigfloor;    // AdjustSigma lower bound (Gaussian)
    R ph0;         // omega * tau0.real reduced to [-pi, pi]
    R omdt;        // omega * dtau.real
    R att0, att1;  // omega * tau0.imag, omega * dtau.imag
    double zmin, zmax;   // receiver depth window of the segment
    int izlo, niz;
};

// Beam-receiver contributions of one segment for one frequency
// (InfluenceGeoCore + ApplyContribution, src/influence.hpp:423-473,897-1024):
// constructed once per (segment, frequency), column() once per receiver
// column, eval() per receiver depth; eval returns false outside the beam window.
// The FP64 policy keeps the reference's operation order. The mixed policy keeps
// the segment constants in registers, uses the per-column constants
// A = dr tx / rlen, Cn = dr tz, folds the Gaussian weight and the attenuation
// into one base-2 exponential, and evaluates the phase with the hardware
// sin/cos after an explicit 2 pi reduction.
template<typename R, bool GAUSS, bool COHERENT> struct Contribution;

template<bool GAUSS, bool COHERENT> struct Contribution<double, GAUSS, COHERENT> {
    const SegRec<double> &S;
    const SegFreq<double> &F;
    double dr;
    __device__ __forceinline__ Contribution(const SegRec<double> &S_, const SegFreq<double> &F_)
        : S(S_), F(F_) {}
    __device__ __forceinline__ void column(double rr) { dr = rr - S.x0r; }
    __device__ __forceinline__ bool eval(float zr_f, float2 &v) const
    {
        double dz = (double)zr_f - S.x0z;
        double s = (dr * S.tx + dz * S.tz) / S.rlen;
        double n1 = fabs(dz * S.tx - dr * S.tz);
        double qF = S.q0 + s * S.dq;
        double sigma = fabs(qF * S.rcp_q0), sig0 = sigma;
        if(GAUSS) sigma = max(sigma, F.sigfloor);
        if(n1 >= (GAUSS ? 4.0 : 1.0) * sigma) return false;
        double cnst = S.cnst_num / sqrt(fabs(qF));
        double wgt;
        if(GAUSS) wgt = exp(FLTD(-0.5) * (n1 / sigma) * (n1 / sigma)) * (sig0 / sigma);
        else wgt = (sigma - n1) / sigma;
        bool caustic = (qF <= 0.0 && S.q0 > 0.0) || (qF >= 0.0 && S.q0 < 0.0);
        double ph = caustic ? S.phase_b : S.phase_a;
        if(COHERENT) {
            double amp = cnst * wgt * exp(F.att0 + s * F.att1);
            double ang = reduce_2pi(F.ph0 + s * F.omdt - ph), sn, cs;
            sincos(ang, &sn, &cs);
            v = make_float2((float)(amp * cs), (float)(-amp * sn));
        } else {
            double vv = cnst * exp(F.att0 + s * F.att1);
            vv = vv * vv * wgt;
            if(GAUSS) vv *= sqrt(FLTD(2.0) * BHCB_PI);
            v = make_float2((float)vv, 0.f);
        }
        return true;
    }
};

// Warp-cooperative influence: each warp stages 32 segment records, then for
// every frequency splits itself into sub-groups of g lanes (g = 4..32, chosen
// from the chunk's average work per segment); a group takes one segment at a
// time, keeps its fields in registers and strides its lanes over the depths of
// each receiver column, so consecutive lanes reduce into consecutive addresses.
template<typename R, bool GAUSS, bool COHERENT> __global__ void __launch_bounds__(32 * WARPS_PER_CTA, 6)
influence_kernel(const SegRec<R> *__restrict__ segs, unsigned long long cap,
                 const GroupDev *__restrict__ groups, int ngroups, const double *__restrict__ freqs,
                 float2 *__restrict__ acc, RunCounters *ctr)
{
    // the trace kernel's slot counter may exceed the capacity on overflow
    const unsigned long long nseg = min(__ldcg(&ctr->nseg), cap);
    __shared__ SegRec<R> s_rec[WARPS_PER_CTA][32];
    __shared__ SegFreq<R> s_sf[WARPS_PER_CTA][32];
    __shared__ long long s_base[WARPS_PER_CTA][32];       // field offset of (isz, ir=0, iz=0), f=0
    __shared__ const double *s_rr[WARPS_PER_CTA][32];
    __shared__ const float *s_rz[WARPS_PER_CTA][32];
    __shared__ long long s_stride[WARPS_PER_CTA][32];     // per-frequency accumulator stride
    __shared__ int s_nrzp[WARPS_PER_CTA][32];             // 0 -> irregular grid
    __shared__ int s_nf[WARPS_PER_CTA][32];               // frequencies of the segment's group
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned long long nchunks = (nseg + 31) / 32;
    unsigned int evals = 0;
    for(;;) {
        // dynamic work queue: chunks differ widely in work
        unsigned long long ch = 0;
        if(lane == 0) ch = atomicAdd(&ctr->chunk_counter, 1ull);
        ch = __shfl_sync(0xffffffffu, ch, 0);
        if(ch >= nchunks) break;
        // segments are stored in trace order, so the last chunks hold the
        // far-range segments with the widest beams: take the heaviest first
        ch = nchunks - 1 - ch;
        {
            const int words = sizeof(SegRec<R>) / 16;
            const uint4 *src = reinterpret_cast<const uint4 *>(segs + ch * 32);
            uint4 *dst = reinterpret_cast<uint4 *>(&s_rec[w][0]);
            int nvalid = (int)min(32ull, nseg - ch * 32);
            for(int k = lane; k < nvalid * words; k += 32) dst[k] = __ldcs(src + k);
            __syncwarp();
            if(lane >= nvalid) s_rec[w][lane].job = -1;
        }
        __syncwarp();
        const SegRec<R> &my = s_rec[w][lane];
        const bool valid = my.job >= 0;
        const EnvDev *e = nullptr;
        int nfreq = 0, freq_base = 0;
        if(valid) {
            const GroupDev &G = groups[find_group(groups, ngroups, my.job)];
            e = G.env;
            nfreq = G.nfreq;
            freq_base = G.freq_base;
            int local = (int)((long long)my.job - G.job_base);
            int nal = e->isingle > 0 ? 1 : e->nalpha;
            int isz = local / nal;
            s_base[w][lane] = G.acc_base + (long long)isz * e->nrr * G.acc_nz;
            s_rr[w][lane] = e->rr;
            s_rz[w][lane] = e->rz;
            s_stride[w][lane] = G.acc_stride_f;
            s_nrzp[w][lane] = e->irregular ? 0 : G.acc_nz;
        }
        s_nf[w][lane] = nfreq;
        int maxf = nfreq;
        for(int o = 16; o > 0; o >>= 1) maxf = max(maxf, __shfl_xor_sync(0xffffffffu, maxf, o));
        for(int f = 0; f < maxf; ++f) {
            int cnt = 0;
            if(valid && f < nfreq) {
                double freq = freqs[freq_base + f];
                double omega = 2.0 * BHCB_PI * freq;
                SegFreq<R> sf;
                R sig = my.sigma_seg;
                sf.sigfloor = (R)0;
                if(GAUSS) {   // AdjustSigma (src/influence.hpp:91-100)
                    R lam = my.c0 / (R)freq;
                    R fl = min((R)FLTD(0.2) * (R)freq * my.tau1r, (R)BHCB_PI * lam);
                    sf.sigfloor = fl;
                    sig = max(sig, fl);
                }
                double rmax = (GAUSS ? 4.0 : 1.0) * (double)sig;
                if(fabs((double)my.tx) > FLTD(0.50001)) {
                    sf.zmin = (double)my.zlo - rmax;
                    sf.zmax = (double)my.zhi + rmax;
                } else {   // steep segment: every depth (src/influence.hpp:1285-1292)
                    sf.zmin = -1.7976931348623157e308;
                    sf.zmax = 1.7976931348623157e308;
                }
                if(e->irregular) {
                    sf.niz = 1;
                    sf.izlo = 0;
                } else {
                    sf.izlo = lower_f(e->rz, e->nrz, sf.zmin);
                    sf.niz = upper_f(e->rz, e->nrz, sf.zmax) - sf.izlo;
                }
                sf.ph0 = (R)reduce_2pi(omega * my.tau0r);
                sf.omdt = (R)(omega * (double)my.dtaur);
                sf.att0 = (R)(omega * (double)my.tau0i);
                sf.att1 = (R)(omega * (double)my.dtaui);
                s_sf[w][lane] = sf;
                cnt = sf.niz > 0 ? (my.ir_hi - my.ir_lo + 1) * sf.niz : 0;
            }
            int tot = cnt;
            for(int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
            if(tot == 0) continue;
            __syncwarp();
            // group size from the average depth-run length of the chunk
            int avg = tot >> 5;
            int g = avg >= 24 ? 32 : avg >= 12 ? 16 : avg >= 6 ? 8 : 4;
            int ngrp = 32 / g, gid = lane / g, lig = lane & (g - 1);
            for(int k = gid; k < 32; k += ngrp) {
                const SegRec<R> &S = s_rec[w][k];
                if(S.job < 0) continue;
                const SegFreq<R> F = s_sf[w][k];
                const long long base = s_base[w][k] + (long long)f * s_stride[w][k];
                const double *rr = s_rr[w][k];
                const float *rz = s_rz[w][k];
                const int nrzp = s_nrzp[w][k];
                if(f >= s_nf[w][k]) continue;   // its group has fewer frequencies
                if(nrzp) {
                    // rectilinear grid: the group walks the flattened (column, depth)
                    // pairs of the segment, depth fastest, so the idle tail is paid
                    // once per segment; a lane recomputes its column constants only
                    // when it moves to the next column.
                    const int niz = F.niz, total = (S.ir_hi - S.ir_lo + 1) * niz;
                    const float *zp = rz + F.izlo;
                    int col = lig / niz, j = lig - col * niz, ccol = -1;
                    Contribution<R, GAUSS, COHERENT> C(S, F);
                    float2 *colp = nullptr;
                    for(int e = lig; e < total; e += g) {
                        if(col != ccol) {
                            ccol = col;
                            int ir = S.ir_lo + col;
                            C.column(rr[ir]);
                            colp = acc + base + (long long)ir * nrzp + F.izlo;
                        }
                        float2 v;
                        if(C.eval(zp[j], v)) {
                            atomicAdd(colp + j, v);
                            ++evals;
                        }
                        j += g;
                        while(j >= niz) { j -= niz; ++col; }
                    }
                } else {
                    // irregular grid: one receiver per column, at depth rz[ir]
                    Contribution<R, GAUSS, COHERENT> C(S, F);
                    for(int ir = S.ir_lo + lig; ir <= S.ir_hi; ir += g) {
                        double zr = (double)rz[ir];
                        if(zr < F.zmin || zr > F.zmax) continue;
                        C.column(rr[ir]);
                        float2 v;
                        if(C.eval(rz[ir], v)) {
                            atomicAdd(acc + base + ir, v);
                            ++evals;
                        }
                    }
                }
            }
            __syncwarp();
        }
    }
    for(int o = 16; o > 0; o >>= 1) evals += __shfl_xor_sync(0xffffffffu, evals, o);
    if(lane == 0 && evals) atomicAdd(&ctr->nevals, (unsigned long long)evals);
}

// ScalePressure (src/influence.hpp:1556-1627, 2-D) fused with the transpose
// acc[f][isz][ir][iz] (rows acc_nz long) -> out[f][isz][iz][ir].
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
        size_t abase = (size_t)G.acc_base + (size_t)plane * nr * G.acc_nz;
        // load: rows ir, contiguous iz
        for(int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
            int ir = tr * 32 + yy, iz = tz * 32 + threadIdx.x;
            if(ir < nr && iz < nz) tile[yy][threadIdx.x] = acc[abase + (size_t)ir * G.acc_nz + iz];
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

__global__ void set_counter_kernel(unsigned long long *p, unsigned long long v) { *p = v; }

// ---------------------------------------------------------------- launchers
cudaError_t launch_set_counter(unsigned long long *p, unsigned long long v, cudaStream_t st)
{
    set_counter_kernel<<<1, 1, 0, st>>>(p, v);
    return cudaGetLastError();
}

template<typename R> cudaError_t launch_trace(const GroupDev *groups, int ngroups, long long njobs,
                                              void *segs, unsigned long long cap, RunCounters *ctr,
                                              unsigned long long *job_counter, unsigned int *blk_state,
                                              int grid, int block, cudaStream_t st, unsigned int stage_bytes,
                                              int lanes)
{
    // the ray state is FP64 in both precisions (the mixed precision writes FP32
    // segment records for its FP32 influence kernel): the trajectory, and with it
    // every step and reflection decision, is the FP64 one
    static bool attr_set = false;
    if(!attr_set) {   // dynamic shared memory above the 48 KB default
        cudaError_t e = cudaFuncSetAttribute(trace_kernel<double, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)STAGE_MAX_BYTES);
        if(e != cudaSuccess) return e;
        attr_set = true;
    }
    if(stage_bytes > STAGE_MAX_BYTES) stage_bytes = STAGE_MAX_BYTES;
    trace_kernel<double, R><<<grid, block, stage_bytes, st>>>(groups, ngroups, njobs, (SegRec<R> *)segs, cap, ctr,
                                                              job_counter, blk_state, stage_bytes, lanes);
    return cudaGetLastError();
}

cudaError_t launch_influence_mixed(const void *segs, unsigned long long cap, const GroupDev *groups, int ngroups,
                                   const double *freqs, float2 *acc, RunCounters *ctr, bool gauss,
                                   bool coherent, int grid, cudaStream_t st, unsigned int *blk_state,
                                   unsigned long long *scan);

template<typename R> cudaError_t launch_influence(const void *segs, unsigned long long nseg,
                                                  const GroupDev *groups, int ngroups,
                                                  const double *freqs, float2 *acc,
                                                  RunCounters *ctr, bool gauss, bool coherent,
                                                  int grid, cudaStream_t st)
{
    if constexpr(sizeof(R) == 4) {
        return launch_influence_mixed(segs, nseg, groups, ngroups, freqs, acc, ctr, gauss, coherent, grid, st,
                                      nullptr, nullptr);
    } else {
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
}

cudaError_t launch_scale(const float2 *acc, float2 *out, const GroupDev *groups, int ngroups,
                         int grid_x, cudaStream_t st)
{
    dim3 block(32, 8), grid(grid_x, 1, ngroups);
    scale_kernel<<<grid, block, 0, st>>>(acc, out, groups, ngroups);
    return cudaGetLastError();
}

template cudaError_t launch_trace<float>(const GroupDev *, int, long long, void *, unsigned long long,
                                         RunCounters *, unsigned long long *, unsigned int *, int, int,
                                         cudaStream_t, unsigned int, int);
template cudaError_t launch_trace<double>(const GroupDev *, int, long long, void *, unsigned long long,
                                          RunCounters *, unsigned long long *, unsigned int *, int, int,
                                          cudaStream_t, unsigned int, int);
template cudaError_t launch_influence<float>(const void *, unsigned long long, const GroupDev *, int,
                                             const double *, float2 *, RunCounters *, bool, bool, int,
                                             cudaStream_t);
template cudaError_t launch_influence<double>(const void *, unsigned long long, const GroupDev *, int,
                                              const double *, float2 *, RunCounters *, bool, bool, int,
                                              cudaStream_t);

size_t seg_record_bytes(bool fp64) { return fp64 ? sizeof(SegRec<double>) : sizeof(SegRec<float>); }

cudaError_t launch_rays(const GroupDev *groups, int ngroups, const long long *jobs, const int *limits, int nitems,
                        const long long *off, double2 *pts, int *npts, int *bnc, RunCounters *ctr, bool count,
                        int sm_count, cudaStream_t st)
{
    if(nitems <= 0) return cudaSuccess;
    int grid = (nitems + 63) / 64;
    if(grid > sm_count * 16) grid = sm_count * 16;
    if(count)
        ray_kernel<true><<<grid, 64, 0, st>>>(groups, ngroups, jobs, limits, nitems, off, pts, npts, bnc, ctr);
    else
        ray_kernel<false><<<grid, 64, 0, st>>>(groups, ngroups, jobs, limits, nitems, off, pts, npts, bnc, ctr);
    return cudaGetLastError();
}

} // namespace bhcb
