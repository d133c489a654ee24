// Mixed-precision influence kernel for sm_100a (BHCB_PREC_MIXED).
//
// Evaluates every beam-receiver contribution of the segments written by the
// trace kernel (InfluenceGeoCore + ApplyContribution, Cartesian hat / Gaussian
// beams, src/influence.hpp:423-473,897-1024) and reduces them into the
// range-major accumulator acc[field][isz][ir][iz].
//
// Work layout. Each warp takes work items from a dynamic queue, heaviest
// first: an item is 32 segments (one chunk of one ray) at one frequency of
// their trace group (beside a running trace, a whole published chunk with all
// its frequencies), so that the heaviest chunk's frequencies spread over
// several warps instead of one warp ending the launch alone. For the item:
// Beside a running trace (blk_state set), a launch takes only the chunks the
// tracer has published and exits when the rest are not ready; the host
// relaunches it until the trace ends (no kernel waits for another).
//   1. prep: lane k turns segment k into a SegFreqM block (window of receiver
//      depths, frequency constants, float column / point constants, the
//      accumulator row pointer) in shared memory;
//   2. the warp splits into groups of g lanes (4..32, from the chunk's mean
//      work); a group walks the flattened (receiver column, depth pair) units of
//      one segment, pairs fastest, so consecutive lanes update consecutive
//      16-byte accumulator words. A pair is the depth indices (2P, 2P+1); its
//      two contributions are computed with Blackwell's paired FP32 operations
//      and added with one 16-byte vector atomic. Irregular receiver grids (one
//      receiver per column) use the scalar form.
// Positions and the travel time's integer part of the phase are FP64 in the
// segment record; the per-contribution math is FP32 with the hardware
// approximations (ex2, rsqrt, rcp, sin, cos), sin/cos after an explicit 2 pi
// reduction.
#include <cuda_runtime.h>

#include "bhcb_internal.h"
#include "device_math.cuh"
#include "trace2d.cuh"
#include "influence2d.cuh"

namespace bhcb {

namespace {

constexpr int MW = 4;   // warps per CTA
constexpr float LOG2E = 1.44269504088896340736f;

// per (segment, frequency) block built by the prep lane
struct alignas(16) SegFreqM {
    float txr, tz, Bz, x0z;      // tx / rlen, tz, tz / rlen, point0 depth
    float tx, dq, q0, rcpq;      // unit tangent x, q1 - q0, q0, Dalpha / c0
    float sfl, sgq, cA, cB;      // sigma floor, sign(q0), phase constants (regular / caustic)
    float omdt, lg0, lg1, cn;    // omega dtau, log2 attenuation (at s = 0, slope), amplitude numerator
    double x0r;                  // point0 range
    float2 *acc;                 // accumulator of this segment's source depth and frequency
    const double *rr;
    const float *rz;
    int ir_lo, ncols;            // receiver columns
    int lo, hi;                  // depth window [lo, hi) (rectilinear) or float bits of [zmin, zmax]
    int p0, npair;               // first depth pair, pairs per column (0: irregular grid)
    uint32_t magic;              // floor((2^32 - 1) / npair) + 1: x / npair = umulhi(x, magic) for x * npair < 2^32 (npair > 1)
    int half_nz;                 // accumulator row length in pairs
    int q, rq;                   // group stride g = q * npair + rq
    int valid, pad;
};

__device__ __forceinline__ int lower_ff(const float *a, int n, float v)   // first a[i] >= v
{
    int lo = 0, hi = n;
    while(lo < hi) {
        int m = (lo + hi) >> 1;
        if(a[m] < v) lo = m + 1; else hi = m;
    }
    return lo;
}
__device__ __forceinline__ int upper_ff(const float *a, int n, float v)   // first a[i] > v
{
    int lo = 0, hi = n;
    while(lo < hi) {
        int m = (lo + hi) >> 1;
        if(a[m] <= v) lo = m + 1; else hi = m;
    }
    return lo;
}

// Builds the block of segment S for one frequency; returns its work units.
template<bool GAUSS> __device__ __forceinline__ int prep_segment(
    const SegRec<float> &S, const GroupDev &G, const EnvDev &e, int f, double freq, float2 *acc, SegFreqM &P)
{
    P.valid = 0;
    // AdjustSigma (src/influence.hpp:91-100) and the depth window of the
    // segment (src/influence.hpp:1285-1292); window bounds in double, compared
    // in float after rounding outward, which selects the same receivers
    float sig = S.sigma_seg, fl = 0.f;
    if(GAUSS) {
        float lam = S.c0 / (float)freq;
        fl = fminf(0.2f * (float)freq * S.tau1r, 3.14159265358979323846f * lam);
        sig = fmaxf(sig, fl);
    }
    double rmax = (GAUSS ? 4.0 : 1.0) * (double)sig;
    double zmin = -1.7976931348623157e308, zmax = 1.7976931348623157e308;
    if(fabs((double)S.tx) > FLTD(0.50001)) {
        zmin = (double)S.zlo - rmax;
        zmax = (double)S.zhi + rmax;
    }
    const float zminf = __double2float_ru(zmin), zmaxf = __double2float_rd(zmax);
    const int ncols = S.ir_hi - S.ir_lo + 1;
    int units;
    int local = (int)((long long)S.job - G.job_base);
    int nal = e.isingle > 0 ? 1 : e.nalpha;
    int isz = local / nal;
    long long base = G.acc_base + (long long)f * G.acc_stride_f + (long long)isz * e.nrr * G.acc_nz;
    P.acc = acc + base;
    if(e.irregular) {
        P.lo = __float_as_int(zminf);
        P.hi = __float_as_int(zmaxf);
        P.npair = 0;
        P.p0 = 0;
        P.magic = 0;
        P.half_nz = 0;
        units = ncols;
    } else {
        int lo = lower_ff(e.rz, e.nrz, zminf), hi = upper_ff(e.rz, e.nrz, zmaxf);
        if(hi <= lo) return 0;
        P.lo = lo;
        P.hi = hi;
        P.p0 = lo >> 1;
        P.npair = ((hi + 1) >> 1) - P.p0;
        P.magic = P.npair > 1 ? (uint32_t)(0xffffffffu / (uint32_t)P.npair) + 1u : 0u;   // npair 1: x / 1 = x
        P.half_nz = G.acc_nz >> 1;
        units = ncols * P.npair;
    }
    const double omega = 2.0 * BHCB_PI * freq;
    const float ph0 = (float)reduce_2pi(omega * S.tau0r);
    const float inv_rlen = 1.0f / S.rlen;
    P.txr = S.tx * inv_rlen;
    P.tz = S.tz;
    P.Bz = S.tz * inv_rlen;
    P.x0z = (float)S.x0z;
    P.tx = S.tx;
    P.dq = S.dq;
    P.q0 = S.q0;
    P.rcpq = S.rcp_q0;
    P.sfl = fl;
    // caustic branch of the phase, (q <= 0 && q0 > 0) || (q >= 0 && q0 < 0),
    // is sign(q0) * q <= 0 with sign(q0) != 0
    P.sgq = S.q0 > 0.f ? 1.f : (S.q0 < 0.f ? -1.f : 0.f);
    P.cA = ph0 - S.phase_a;
    P.cB = P.sgq != 0.f ? ph0 - S.phase_b : P.cA;
    P.omdt = (float)(omega * (double)S.dtaur);
    P.lg0 = (float)(omega * (double)S.tau0i) * LOG2E;
    P.lg1 = (float)(omega * (double)S.dtaui) * LOG2E;
    P.cn = S.cnst_num;
    P.x0r = S.x0r;
    P.rr = e.rr;
    P.rz = e.rz;
    P.ir_lo = S.ir_lo;
    P.ncols = ncols;
    P.valid = 1;
    return units;
}

// -round(a / 2 pi) by the 1.5 * 2^23 shifter (|a| << 2^22), then a mod 2 pi
__device__ __forceinline__ float2 reduce_2pi_pair(float2 a)
{
    const float SH = 12582912.f, I2P = 0.159154943f;
    const float2 nk = __fadd2_rn(__ffma2_rn(a, make_float2(-I2P, -I2P), make_float2(-SH, -SH)),
                                 make_float2(SH, SH));
    a = __ffma2_rn(nk, make_float2(6.28318548f, 6.28318548f), a);
    return __ffma2_rn(nk, make_float2(-1.7484555e-7f, -1.7484555e-7f), a);
}

// Two receivers of one column (depths zr.x, zr.y); ok0 / ok1: inside the
// depth window. A = dr tx / rlen, Cn = dr tz are the column constants.
template<bool GAUSS, bool COHERENT> __device__ __forceinline__ int eval_pair(
    const SegFreqM &P, float A, float Cn, float2 zr, bool ok0, bool ok1, float4 &v)
{
    const float2 dz = __fadd2_rn(zr, make_float2(-P.x0z, -P.x0z));
    const float2 s = __ffma2_rn(dz, make_float2(P.Bz, P.Bz), make_float2(A, A));
    const float2 nr = __ffma2_rn(dz, make_float2(P.tx, P.tx), make_float2(-Cn, -Cn));
    const float2 qF = __ffma2_rn(s, make_float2(P.dq, P.dq), make_float2(P.q0, P.q0));
    const float2 sq = __fmul2_rn(qF, make_float2(P.rcpq, P.rcpq));
    const float n0 = fabsf(nr.x), n1 = fabsf(nr.y);
    const float g0 = fabsf(sq.x), g1 = fabsf(sq.y);
    const float sg0 = GAUSS ? fmaxf(g0, P.sfl) : g0, sg1 = GAUSS ? fmaxf(g1, P.sfl) : g1;
    const float W = GAUSS ? 4.f : 1.f;
    const bool in0 = ok0 && !(n0 >= W * sg0), in1 = ok1 && !(n1 >= W * sg1);
    if(!(in0 || in1)) return 0;
    const float2 rs = make_float2(rcp_ftz(sg0), rcp_ftz(sg1));
    float2 lg = __ffma2_rn(s, make_float2(P.lg1, P.lg1), make_float2(P.lg0, P.lg0));
    if(!COHERENT) lg = __fadd2_rn(lg, lg);
    float2 w;
    if(GAUSS) {
        const float2 a = __fmul2_rn(make_float2(n0, n1), rs);
        lg = __ffma2_rn(__fmul2_rn(a, a), make_float2(-0.5f * LOG2E, -0.5f * LOG2E), lg);
        w = __fmul2_rn(make_float2(g0, g1), rs);
    } else {
        w = __fmul2_rn(make_float2(sg0 - n0, sg1 - n1), rs);
    }
    const float2 r = make_float2(rsqrt_ftz(fabsf(qF.x)), rsqrt_ftz(fabsf(qF.y)));
    const float2 e = make_float2(ex2_ftz(lg.x), ex2_ftz(lg.y));
    if(COHERENT) {
        float2 amp = __fmul2_rn(__fmul2_rn(r, w), __fmul2_rn(e, make_float2(P.cn, P.cn)));
        amp.x = in0 ? amp.x : 0.f;
        amp.y = in1 ? amp.y : 0.f;
        const float2 sgn = __fmul2_rn(qF, make_float2(P.sgq, P.sgq));
        float2 ang = __ffma2_rn(s, make_float2(P.omdt, P.omdt),
                                make_float2(sgn.x <= 0.f ? P.cB : P.cA, sgn.y <= 0.f ? P.cB : P.cA));
        ang = reduce_2pi_pair(ang);
        const float2 cs = make_float2(cos_ftz(ang.x), cos_ftz(ang.y));
        const float2 sn = make_float2(sin_ftz(ang.x), sin_ftz(ang.y));
        const float2 re = __fmul2_rn(amp, cs);
        const float2 im = __fmul2_rn(make_float2(-amp.x, -amp.y), sn);
        v = make_float4(re.x, im.x, re.y, im.y);
    } else {
        const float k = GAUSS ? P.cn * P.cn * 2.50662827463100050242f : P.cn * P.cn;   // sqrt(2 pi)
        const float2 vv = __fmul2_rn(__fmul2_rn(__fmul2_rn(r, r), w), __fmul2_rn(e, make_float2(k, k)));
        v = make_float4(in0 ? vv.x : 0.f, 0.f, in1 ? vv.y : 0.f, 0.f);
    }
    return (int)in0 + (int)in1;
}

// one receiver (irregular grid)
template<bool GAUSS, bool COHERENT> __device__ __forceinline__ bool eval_one(
    const SegFreqM &P, float A, float Cn, float zr, float2 &v)
{
    const float dz = zr - P.x0z;
    const float s = fmaf(dz, P.Bz, A);
    const float n1 = fabsf(fmaf(dz, P.tx, -Cn));
    const float qF = fmaf(s, P.dq, P.q0);
    const float sig0 = fabsf(qF * P.rcpq);
    const float sigma = GAUSS ? fmaxf(sig0, P.sfl) : sig0;
    if(n1 >= (GAUSS ? 4.f : 1.f) * sigma) return false;
    const float rs = rcp_ftz(sigma);
    const float la = fmaf(s, P.lg1, P.lg0);
    float lgs = 0.f, w;
    if(GAUSS) {
        const float a = n1 * rs;
        lgs = (a * a) * (-0.5f * LOG2E);
        w = sig0 * rs;
    } else {
        w = (sigma - n1) * rs;
    }
    const float cnst = P.cn * rsqrt_ftz(fabsf(qF));
    if(COHERENT) {
        const float amp = cnst * w * ex2_ftz(la + lgs);
        const float2 ang = reduce_2pi_pair(make_float2(fmaf(s, P.omdt, P.sgq * qF <= 0.f ? P.cB : P.cA), 0.f));
        v = make_float2(amp * cos_ftz(ang.x), -amp * sin_ftz(ang.x));
    } else {
        float vv = cnst * cnst * w * ex2_ftz(la + la + lgs);
        if(GAUSS) vv *= 2.50662827463100050242f;
        v = make_float2(vv, 0.f);
    }
    return true;
}

// At most 64 registers per thread (8 CTAs per SM): the extra resident warps
// hide more latency than the few spilled values cost (measured 8 % faster on
// the 20001-ray Gaussian workload than at 96 registers; 48 spills in the
// pair loop and is slower).
template<bool GAUSS, bool COHERENT> __global__ void __launch_bounds__(32 * MW, 8)
influence_kernel_mixed(const SegRec<float> *__restrict__ segs, unsigned long long cap,
                       const GroupDev *__restrict__ groups, int ngroups, const double *__restrict__ freqs,
                       float2 *__restrict__ acc, RunCounters *ctr, unsigned int *blk_state,
                       unsigned long long *scan)
{
    // the trace kernel's slot counter may exceed the capacity on overflow
    const unsigned long long nseg = min(__ldcg(&ctr->nseg), cap);
    unsigned long long *queue = scan ? scan : &ctr->chunk_counter;
    __shared__ SegFreqM s_p[MW][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned long long nchunks = (nseg + 31) / 32;
    // frequencies per chunk: items are (chunk, frequency) pairs, except beside
    // a running trace, where an item is a whole published chunk
    int fsplit = 0;
    if(!blk_state) {
        for(int g = lane; g < ngroups; g += 32) fsplit = max(fsplit, groups[g].nfreq);
        for(int o = 16; o > 0; o >>= 1) fsplit = max(fsplit, __shfl_xor_sync(0xffffffffu, fsplit, o));
        fsplit = max(fsplit, 1);
    }
    const unsigned long long nitems = fsplit ? nchunks * (unsigned long long)fsplit : nchunks;
    unsigned int evals = 0;
    for(;;) {
        unsigned long long it = 0;
        if(lane == 0) it = atomicAdd(queue, 1ull);
        it = __shfl_sync(0xffffffffu, it, 0);
        if(it >= nitems) break;
        // segments are stored in trace order, so the last chunks hold the
        // far-range segments with the widest beams: take the heaviest first
        it = nitems - 1 - it;
        const unsigned long long ch = fsplit ? it / (unsigned long long)fsplit : it;
        const int fsel = fsplit ? (int)(it - ch * (unsigned long long)fsplit) : -1;
        if(blk_state) {
            // running beside the trace: take a chunk (a 32-slot block of one
            // ray) only once the tracer has published it; skipped blocks are
            // taken by a later launch
            unsigned int got = 0;
            if(lane == 0) got = atomicCAS(&blk_state[ch], 1u, 2u);
            got = __shfl_sync(0xffffffffu, got, 0);
            if(got != 1u) continue;
            __threadfence();
        }
        const unsigned long long k0 = ch * 32 + lane;
        const bool have = k0 < nseg;
        SegRec<float> my;
        if(have) {
            const uint4 *src = reinterpret_cast<const uint4 *>(segs + k0);
            uint4 *dst = reinterpret_cast<uint4 *>(&my);
#pragma unroll
            for(int i = 0; i < (int)(sizeof(SegRec<float>) / 16); ++i) dst[i] = __ldcg(src + i);
        } else {
            my.job = -1;
        }
        const bool valid = my.job >= 0;
        int gi = 0, nfreq = 0;
        if(valid) {
            gi = find_group(groups, ngroups, my.job);
            nfreq = groups[gi].nfreq;
        }
        int maxf = nfreq;
        for(int o = 16; o > 0; o >>= 1) maxf = max(maxf, __shfl_xor_sync(0xffffffffu, maxf, o));
        const int f0 = fsel >= 0 ? fsel : 0, f1 = fsel >= 0 ? min(fsel + 1, maxf) : maxf;
        for(int f = f0; f < f1; ++f) {
            int cnt = 0;
            SegFreqM &mine = s_p[w][lane];
            if(valid && f < nfreq) {
                const GroupDev &G = groups[gi];
                cnt = prep_segment<GAUSS>(my, G, *G.env, f, freqs[G.freq_base + f], acc, mine);
            } else {
                mine.valid = 0;
            }
            int tot = cnt;
            for(int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
            if(tot == 0) {
                __syncwarp();
                continue;
            }
            // group size from the mean work units of the chunk
            const int avg = tot >> 5;
            const int g = avg >= 24 ? 32 : avg >= 12 ? 16 : avg >= 6 ? 8 : 4;
            if(mine.valid && mine.npair) {
                const int q = mine.npair > 1 ? (int)__umulhi((uint32_t)g, mine.magic) : g;
                mine.q = q;
                mine.rq = g - q * mine.npair;
            }
            __syncwarp();
            const int ngrp = 32 / g, gid = lane / g, lig = lane & (g - 1);
            for(int k = gid; k < 32; k += ngrp) {
                const SegFreqM P = s_p[w][k];   // register copy: the pair loop reads it every iteration
                if(!P.valid) continue;
                if(P.npair) {
                    // rectilinear grid: flattened (column, depth pair) units
                    const int npair = P.npair, ncols = P.ncols, q = P.q, rq = P.rq;
                    const int lo = P.lo, hi = P.hi, p0 = P.p0;
                    const float2 *zp2 = reinterpret_cast<const float2 *>(P.rz) + p0;
                    float4 *const acc4 = reinterpret_cast<float4 *>(P.acc) + p0;
                    const long long rowstep = P.half_nz;
                    int col = npair > 1 ? (int)__umulhi((uint32_t)lig, P.magic) : lig;
                    int jp = lig - col * npair, ccol = -1;
                    float A = 0.f, Cn = 0.f;
                    float4 *colp = acc4;
                    while(col < ncols) {
                        if(col != ccol) {
                            ccol = col;
                            const int ir = P.ir_lo + col;
                            const float dr = (float)(P.rr[ir] - P.x0r);
                            A = dr * P.txr;
                            Cn = dr * P.tz;
                            colp = acc4 + (long long)ir * rowstep;
                        }
                        const int d0 = 2 * (p0 + jp);
                        float4 v;
                        const int n = eval_pair<GAUSS, COHERENT>(P, A, Cn, zp2[jp], d0 >= lo, d0 + 1 < hi, v);
                        if(n) {
                            atomicAdd(colp + jp, v);
                            evals += n;
                        }
                        jp += rq;
                        col += q;
                        if(jp >= npair) {
                            jp -= npair;
                            ++col;
                        }
                    }
                } else {
                    // irregular grid: one receiver per column, at depth rz[ir]
                    const float zminf = __int_as_float(P.lo), zmaxf = __int_as_float(P.hi);
                    for(int c = lig; c < P.ncols; c += g) {
                        const int ir = P.ir_lo + c;
                        const float zr = P.rz[ir];
                        if(!(zr >= zminf && zr <= zmaxf)) continue;
                        const float dr = (float)(P.rr[ir] - P.x0r);
                        float2 v;
                        if(eval_one<GAUSS, COHERENT>(P, dr * P.txr, dr * P.tz, zr, v)) {
                            atomicAdd(P.acc + ir, v);
                            ++evals;
                        }
                    }
                }
            }
            __syncwarp();   // s_p is rewritten for the next frequency
        }
    }
    for(int o = 16; o > 0; o >>= 1) evals += __shfl_xor_sync(0xffffffffu, evals, o);
    if(lane == 0 && evals) atomicAdd(&ctr->nevals, (unsigned long long)evals);
}

} // namespace

cudaError_t launch_influence_mixed(const void *segs, unsigned long long cap, const GroupDev *groups, int ngroups,
                                   const double *freqs, float2 *acc, RunCounters *ctr, bool gauss,
                                   bool coherent, int grid, cudaStream_t st, unsigned int *blk_state,
                                   unsigned long long *scan)
{
    const SegRec<float> *s = (const SegRec<float> *)segs;
    const int block = 32 * MW;
    if(gauss && coherent)
        influence_kernel_mixed<true, true><<<grid, block, 0, st>>>(s, cap, groups, ngroups, freqs, acc, ctr,
                                                                   blk_state, scan);
    else if(gauss)
        influence_kernel_mixed<true, false><<<grid, block, 0, st>>>(s, cap, groups, ngroups, freqs, acc, ctr,
                                                                    blk_state, scan);
    else if(coherent)
        influence_kernel_mixed<false, true><<<grid, block, 0, st>>>(s, cap, groups, ngroups, freqs, acc, ctr,
                                                                    blk_state, scan);
    else
        influence_kernel_mixed<false, false><<<grid, block, 0, st>>>(s, cap, groups, ngroups, freqs, acc, ctr,
                                                                     blk_state, scan);
    return cudaGetLastError();
}

} // namespace bhcb
