// Tiled influence kernel of the mixed-precision TL path (sm_100a).
//
// Evaluates the beam-receiver contributions of the segments the trace kernel
// wrote (InfluenceGeoCore + ApplyContribution, Cartesian hat / Gaussian beams,
// src/influence.hpp:423-473,897-1024) receiver-tile by receiver-tile instead of
// segment by segment:
//
//   1. tile_bin_kernel (count): every segment adds itself to the bins of the
//      column blocks (TILE_COLS receiver ranges) its receiver columns touch,
//      with an estimate of its work there;
//   2. tile_scan_kernel (one CTA): bin offsets, the fill cursors, and the tile
//      order (heaviest estimated work first, in log2 buckets);
//   3. tile_bin_kernel (fill): the segment indices into each bin's list;
//   4. tile_kernel: persistent CTAs take (bin, depth block) tiles from the
//      queue. Thread t owns receiver depth db * TILE_DEPTHS + t and the tile's
//      TILE_COLS ranges, and keeps the complex field of every frequency of the
//      group in registers while the CTA walks the bin's segments, so no
//      contribution goes through an atomic. The tile is written once, scaled
//      (ScalePressure, src/influence.hpp:1556-1627) and in the reference layout
//      [field][isz][iz][ir] (GetFieldAddr, src/common.hpp:393-405).
//
// Per segment and frequency, a prep thread computes the frequency constants
// (the phase at the segment start reduced mod 2 pi in FP64, the attenuation
// and phase slopes, the Gaussian width floor of AdjustSigma and the depth
// window of src/influence.hpp:1285-1292 rounded outward to float). Per
// receiver column the geometry (s, normal distance, q, beam width) is shared by
// all frequencies; per (column, frequency) the weight and attenuation take one
// base-2 exponential, and on equally spaced ranges the phase of the next
// column is the previous one turned by a per-(segment, frequency) rotation
// instead of a new sine and cosine.
#include <cuda_runtime.h>

#include "bhcb_internal.h"
#include "device_math.cuh"
#include "trace2d.cuh"
#include "influence2d.cuh"

namespace bhcb {

namespace {

constexpr float LOG2E = 1.44269504088896340736f;
constexpr int PB = 128;            // segments prepared per batch
constexpr int NFP_MAX = 10;        // frequencies per pass held in registers

// Prepared segment for one tile (shared memory).
template<int NFP> struct alignas(16) TilePrep {
    float txr, tz, Bz, x0z;        // tx / rlen, tz, tz / rlen, point0 depth
    float tx, dq, q0, rcpq;        // unit tangent x, q1 - q0, q0, Dalpha / c0
    float sgq, cn, kdr, kdi;       // sign(q0), amplitude numerator, e^{i (cB - cA)} of the caustic branch
    float dr[TILE_COLS];           // rr[ir] - point0 range, per tile column
    int dlo, dhi, clo, chi;        // depth window [dlo, dhi) over all frequencies; columns [clo, chi]
    float4 fa[NFP];                // cA (phase at s = 0), omega dtau_r, log2 attenuation at s = 0 and its slope
    float4 fb[NFP];                // width floor, its reciprocal, depth window [zmin, zmax]
    float2 fr[NFP];                // phase rotation from one column to the next (equal range spacing)
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

__device__ __forceinline__ int find_tgroup(const TileGroupDev *tg, int ngroups, int64_t bin)
{
    int lo = 0, hi = ngroups - 1;
    while(lo < hi) {
        int m = (lo + hi + 1) >> 1;
        if(tg[m].bin_base <= bin) lo = m; else hi = m - 1;
    }
    return lo;
}

// --------------------------------------------------------------- binning
// The tail of a segment record: ir_lo, ir_hi, job, is (16-byte aligned).
__device__ __forceinline__ int4 seg_tail(const SegRec<float> *segs, unsigned long long k)
{
    return __ldcg(reinterpret_cast<const int4 *>(&segs[k].ir_lo));
}

template<bool FILL> __global__ void __launch_bounds__(256) tile_bin_kernel(
    const SegRec<float> *__restrict__ segs, unsigned long long cap, const RunCounters *ctr,
    const GroupDev *__restrict__ groups, int ngroups, const TileGroupDev *__restrict__ tg,
    unsigned int *cnt, float *work, unsigned int *list, unsigned long long list_cap)
{
    const unsigned long long nseg = min(__ldcg(&ctr->nseg), cap);
    for(unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < nseg;
        k += (unsigned long long)gridDim.x * blockDim.x) {
        const int4 t = seg_tail(segs, k);
        const int job = t.z;
        if(job < 0) continue;   // unused slot of a ray's 32-slot block
        const int gi = find_group(groups, ngroups, job);
        const GroupDev &G = groups[gi];
        const EnvDev &e = *G.env;
        const int nal = e.isingle > 0 ? 1 : e.nalpha;
        const int isz = (int)(job - G.job_base) / nal;
        const TileGroupDev &T = tg[gi];
        const int cb0 = t.x / TILE_COLS, cb1 = t.y / TILE_COLS;
        float w = 0.f;
        if(!FILL) {
            // work estimate for the tile order only: columns x depths in the
            // window widened by the segment's beam width
            const SegRec<float> &S = segs[k];
            const float halfw = (e.gaussian ? 4.f : 1.f) * S.sigma_seg;
            const float nd = fminf((float)e.nrz, 1.f + (S.zhi - S.zlo + 2.f * halfw) / T.dz_mean);
            w = nd;
        }
        for(int cb = cb0; cb <= cb1; ++cb) {
            const long long bin = T.bin_base + (long long)isz * T.ncb + cb;
            if(FILL) {
                const unsigned int pos = atomicAdd(&cnt[bin], 1u);
                if(pos < list_cap) list[pos] = (unsigned int)k;
            } else {
                const int c0 = max(t.x, cb * TILE_COLS), c1 = min(t.y, cb * TILE_COLS + TILE_COLS - 1);
                atomicAdd(&cnt[bin], 1u);
                atomicAdd(&work[bin], w * (float)(c1 - c0 + 1));
            }
        }
    }
}

// One CTA: exclusive scan of the bin counts into off[0..nbins] and the fill
// cursors (cnt), and the tile order. Tiles are (bin, depth block) pairs coded
// bin * ndb_max + db; they are bucketed by floor(log2(work)) so that the
// persistent tile kernel starts with the heaviest.
constexpr int SCAN_THREADS = 1024;
constexpr int NBUCKET = 40;
// cnt, off and work point at the launch's first bin bin0; nbins bins follow.
__global__ void __launch_bounds__(SCAN_THREADS) tile_scan_kernel(
    unsigned int *cnt, unsigned int *off, const float *work, long long bin0, long long nbins, int ndb_max,
    unsigned int *order, unsigned long long list_cap, RunCounters *ctr)
{
    __shared__ unsigned int s_warp[SCAN_THREADS / 32];
    __shared__ unsigned int s_carry;
    __shared__ unsigned int s_hist[NBUCKET];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if(tid == 0) s_carry = 0;
    if(tid < NBUCKET) s_hist[tid] = 0;
    __syncthreads();
    for(long long base = 0; base < nbins; base += SCAN_THREADS) {
        const long long i = base + tid;
        const unsigned int v = i < nbins ? cnt[i] : 0u;
        unsigned int x = v;
        for(int o = 1; o < 32; o <<= 1) {
            const unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
            if(lane >= o) x += y;
        }
        if(lane == 31) s_warp[wid] = x;
        __syncthreads();
        if(wid == 0) {
            unsigned int y = s_warp[lane];
            for(int o = 1; o < 32; o <<= 1) {
                const unsigned int z = __shfl_up_sync(0xffffffffu, y, o);
                if(lane >= o) y += z;
            }
            s_warp[lane] = y;
        }
        __syncthreads();
        const unsigned int excl = s_carry + (wid ? s_warp[wid - 1] : 0u) + x - v;
        if(i < nbins) {
            off[i] = excl;
            cnt[i] = excl;   // fill cursor
            const float w = work[i];
            const int b = w > 1.f ? min(NBUCKET - 1, (int)log2f(w)) : 0;
            atomicAdd(&s_hist[NBUCKET - 1 - b], (unsigned int)ndb_max);   // heaviest bucket first
        }
        __syncthreads();
        if(tid == SCAN_THREADS - 1) s_carry = excl + v;
        __syncthreads();
    }
    if(tid == 0) {
        off[nbins] = s_carry;
        if(s_carry > list_cap) {
            ctr->nlist = s_carry;
            atomicOr(&ctr->err_bits, 1u << ERR_LIST_OVERFLOW);
        }
        unsigned int run = 0;   // bucket start offsets
        for(int b = 0; b < NBUCKET; ++b) {
            const unsigned int h = s_hist[b];
            s_hist[b] = run;
            run += h;
        }
    }
    __syncthreads();
    // scatter the tiles into their buckets (order within a bucket: roughly by bin)
    for(long long base = 0; base < nbins; base += SCAN_THREADS) {
        const long long i = base + tid;
        if(i < nbins) {
            const float w = work[i];
            const int b = w > 1.f ? min(NBUCKET - 1, (int)log2f(w)) : 0;
            const unsigned int p = atomicAdd(&s_hist[NBUCKET - 1 - b], (unsigned int)ndb_max);
            for(int d = 0; d < ndb_max; ++d) order[p + d] = (unsigned int)((bin0 + i) * ndb_max + d);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ tiles
// Prepares segment S for the tile's columns [ir0, ir0 + ncols) and the
// frequencies [f0, f0 + nf) of its group; returns false if no receiver of the
// tile's depth block lies in its depth window.
template<int NFP, bool GAUSS> __device__ __forceinline__ void tile_prep(
    const SegRec<float> &S, const EnvDev &e, const TileGroupDev &T, const double *freqs, int nf, int ir0,
    int ncols, TilePrep<NFP> &P)
{
    P.clo = max(S.ir_lo, ir0) - ir0;
    P.chi = min(S.ir_hi, ir0 + ncols - 1) - ir0;
    const float inv_rlen = 1.0f / S.rlen;
    P.txr = S.tx * inv_rlen;
    P.tz = S.tz;
    P.Bz = S.tz * inv_rlen;
    P.x0z = (float)S.x0z;
    P.tx = S.tx;
    P.dq = S.dq;
    P.q0 = S.q0;
    P.rcpq = S.rcp_q0;
    // caustic branch of FinalPhase, (q <= 0 && q0 > 0) || (q >= 0 && q0 < 0),
    // is sign(q0) * q <= 0 with sign(q0) != 0; its phase constant differs from
    // the regular one by phase_a - phase_b
    P.sgq = S.q0 > 0.f ? 1.f : (S.q0 < 0.f ? -1.f : 0.f);
    P.cn = S.cnst_num;
    if(P.sgq != 0.f) {
        float sd, cd;
        sincosf(S.phase_a - S.phase_b, &sd, &cd);
        P.kdr = cd;
        P.kdi = sd;
    } else {
        P.kdr = 1.f;
        P.kdi = 0.f;
    }
#pragma unroll
    for(int c = 0; c < TILE_COLS; ++c) P.dr[c] = c < ncols ? (float)(e.rr[ir0 + c] - S.x0r) : 0.f;
    // per frequency: AdjustSigma floor (src/influence.hpp:91-100) and the depth
    // window of the segment (src/influence.hpp:1285-1292), in double, then
    // rounded outward to float, which selects the same receivers as the
    // double comparison
    const bool steep = fabs((double)S.tx) > FLTD(0.50001);
    float zlo_u = 3.4e38f, zhi_u = -3.4e38f;
    const float step = T.uniform_r ? (float)T.rstep * P.txr : 0.f;   // s per column
#pragma unroll
    for(int k = 0; k < NFP; ++k) {
        if(k >= nf) {
            P.fa[k] = make_float4(0.f, 0.f, 0.f, 0.f);
            P.fb[k] = make_float4(0.f, 0.f, 1.f, -1.f);   // empty window
            P.fr[k] = make_float2(1.f, 0.f);
            continue;
        }
        const double freq = freqs[k];
        float sig = S.sigma_seg, fl = 0.f;
        if(GAUSS) {
            const float lam = S.c0 / (float)freq;
            fl = fminf(0.2f * (float)freq * S.tau1r, 3.14159265358979323846f * lam);
            sig = fmaxf(sig, fl);
        }
        const double rmax = (GAUSS ? 4.0 : 1.0) * (double)sig;
        float zminf = -3.4028235e38f, zmaxf = 3.4028235e38f;
        if(steep) {
            zminf = __double2float_ru((double)S.zlo - rmax);
            zmaxf = __double2float_rd((double)S.zhi + rmax);
        }
        zlo_u = fminf(zlo_u, zminf);
        zhi_u = fmaxf(zhi_u, zmaxf);
        const double omega = 2.0 * BHCB_PI * freq;
        const float ph0 = (float)reduce_2pi(omega * S.tau0r);
        const float omdt = (float)(omega * (double)S.dtaur);
        P.fa[k] = make_float4(ph0 - S.phase_a, omdt, (float)(omega * (double)S.tau0i) * LOG2E,
                              (float)(omega * (double)S.dtaui) * LOG2E);
        P.fb[k] = make_float4(fl, GAUSS ? rcp_ftz(fl) : 0.f, zminf, zmaxf);
        float sr, cr;
        sincosf(reduce_2pi(omdt * step), &sr, &cr);
        P.fr[k] = make_float2(cr, sr);
    }
    if(e.irregular) {   // not taken: the tiled path runs on rectilinear grids only
        P.dlo = P.dhi = 0;
        return;
    }
    P.dlo = lower_ff(e.rz, e.nrz, zlo_u);
    P.dhi = upper_ff(e.rz, e.nrz, zhi_u);
}

// Complex accumulator of one (column, frequency) receiver.
struct Acc2 {
    float r, i;
};

template<int NFP, bool GAUSS, bool COHERENT> __global__ void __launch_bounds__(TILE_DEPTHS, 1)
tile_kernel(const SegRec<float> *__restrict__ segs, const GroupDev *__restrict__ groups, int ngroups,
            const TileGroupDev *__restrict__ tg, const double *__restrict__ freqs,
            const unsigned int *__restrict__ list, const unsigned int *__restrict__ off,
            const unsigned int *__restrict__ order, unsigned long long ntiles, int ndb_max,
            unsigned long long list_cap, float2 *__restrict__ out, RunCounters *ctr)
{
    // lists that did not fit were cut short by the fill: the host grows them and runs again
    if(__ldcg(&ctr->err_bits) & (1u << ERR_LIST_OVERFLOW)) return;
    extern __shared__ __align__(16) unsigned char s_dyn[];   // PB prepared segments
    TilePrep<NFP> *s_prep = reinterpret_cast<TilePrep<NFP> *>(s_dyn);
    __shared__ unsigned long long s_tile;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    unsigned int evals = 0;
    for(;;) {
        if(tid == 0) s_tile = atomicAdd(&ctr->tile_counter, 1ull);
        __syncthreads();
        const unsigned long long it = s_tile;
        __syncthreads();   // s_tile is rewritten on the next pass
        if(it >= ntiles) break;
        const unsigned int code = order[it];
        const long long bin = code / ndb_max;
        const int db = (int)(code - bin * ndb_max);
        const int gi = find_tgroup(tg, ngroups, bin);
        const TileGroupDev &T = tg[gi];
        if(db >= T.ndb) continue;   // this group has fewer depth blocks
        const GroupDev &G = groups[gi];
        const EnvDev &e = *G.env;
        const long long lb = bin - T.bin_base;
        const int isz = (int)(lb / T.ncb), cb = (int)(lb - (long long)isz * T.ncb);
        const int ir0 = cb * TILE_COLS, ncols = min(TILE_COLS, e.nrr - ir0);
        const int nz = e.nrz_per_range;
        const int d = db * TILE_DEPTHS + tid;
        const bool have_d = d < nz;
        const float zr = have_d ? e.rz[d] : 0.f;
        const int wd0 = db * TILE_DEPTHS + wid * 32;   // first depth of this warp
        const unsigned int l0 = off[bin], l1 = (unsigned int)min((unsigned long long)off[bin + 1], list_cap);
        for(int f0 = 0; f0 < G.nfreq; f0 += NFP) {
            const int nf = min(NFP, G.nfreq - f0);
            const double *fq = freqs + G.freq_base + f0;
            Acc2 acc[TILE_COLS][NFP];
#pragma unroll
            for(int c = 0; c < TILE_COLS; ++c)
#pragma unroll
                for(int k = 0; k < NFP; ++k) acc[c][k] = Acc2{0.f, 0.f};
            for(unsigned int b0 = l0; b0 < l1; b0 += PB) {
                const int nb = (int)min((unsigned int)PB, l1 - b0);
                __syncthreads();   // the previous batch is consumed
                if(tid < nb) {
                    const SegRec<float> S = segs[list[b0 + tid]];
                    tile_prep<NFP, GAUSS>(S, e, T, fq, nf, ir0, ncols, s_prep[tid]);
                }
                __syncthreads();
                for(int j0 = 0; j0 < nb; j0 += 32) {
                    // segments of these 32 whose depth window meets this warp's depths
                    bool hit = false;
                    if(j0 + lane < nb) {
                        const int lo = s_prep[j0 + lane].dlo, hi = s_prep[j0 + lane].dhi;
                        hit = lo < hi && lo < wd0 + 32 && hi > wd0;
                    }
                    unsigned int mask = __ballot_sync(0xffffffffu, hit);
                    while(mask) {
                        const int j = j0 + __ffs(mask) - 1;
                        mask &= mask - 1;
                        const TilePrep<NFP> &P = s_prep[j];
                        if(!(have_d && d >= P.dlo && d < P.dhi)) continue;
                        // geometry per column, shared by every frequency
                        const float dz = zr - P.x0z;
                        float s[TILE_COLS], n[TILE_COLS], g[TILE_COLS], amp0[TILE_COLS], rg[TILE_COLS];
                        bool br[TILE_COLS];
#pragma unroll
                        for(int c = 0; c < TILE_COLS; ++c) {
                            const float A = P.dr[c] * P.txr, Cn = P.dr[c] * P.tz;
                            s[c] = fmaf(dz, P.Bz, A);
                            n[c] = fabsf(fmaf(dz, P.tx, -Cn));
                            const float qF = fmaf(s[c], P.dq, P.q0);
                            g[c] = fabsf(qF * P.rcpq);
                            rg[c] = rcp_ftz(g[c]);
                            const float r = rsqrt_ftz(fabsf(qF));
                            amp0[c] = COHERENT ? r * P.cn : r * r;
                            br[c] = P.sgq * qF <= 0.f;
                        }
                        const int c0 = P.clo;
                        const bool rot_ok = T.uniform_r;
#pragma unroll
                        for(int k = 0; k < NFP; ++k) {
                            if(k >= nf) break;
                            const float4 fa = P.fa[k], fb = P.fb[k];
                            const float2 fr = P.fr[k];
                            const bool okz = zr >= fb.z && zr <= fb.w;
                            if(!okz) continue;
                            float rr_ = 0.f, ri_ = 0.f;   // e^{i ang} of the current column (branch A)
#pragma unroll
                            for(int c = 0; c < TILE_COLS; ++c) {
                                if(c < c0 || c > P.chi) continue;
                                if(COHERENT) {
                                    if(c == c0 || !rot_ok) {
                                        float ang = fmaf(s[c], fa.y, fa.x);
                                        ang = reduce_2pi(ang);
                                        rr_ = cos_ftz(ang);
                                        ri_ = sin_ftz(ang);
                                    } else {
                                        const float t = rr_ * fr.x - ri_ * fr.y;
                                        ri_ = fmaf(rr_, fr.y, ri_ * fr.x);
                                        rr_ = t;
                                    }
                                }
                                const float sg = GAUSS ? fmaxf(g[c], fb.x) : g[c];
                                if(n[c] >= (GAUSS ? 4.f : 1.f) * sg) continue;
                                const float rs = GAUSS ? (g[c] >= fb.x ? rg[c] : fb.y) : rg[c];
                                float lg = fmaf(s[c], fa.w, fa.z);
                                if(!COHERENT) lg += lg;
                                float w;
                                if(GAUSS) {
                                    const float a = n[c] * rs;
                                    lg = fmaf(a * a, -0.5f * LOG2E, lg);
                                    w = g[c] * rs;
                                } else {
                                    w = (sg - n[c]) * rs;
                                }
                                const float amp = amp0[c] * w * ex2_ftz(lg);
                                if(COHERENT) {
                                    float vr = rr_, vi = ri_;
                                    if(br[c]) {   // caustic branch: turn by e^{i (cB - cA)}
                                        vr = rr_ * P.kdr - ri_ * P.kdi;
                                        vi = fmaf(rr_, P.kdi, ri_ * P.kdr);
                                    }
                                    acc[c][k].r = fmaf(amp, vr, acc[c][k].r);
                                    acc[c][k].i = fmaf(-amp, vi, acc[c][k].i);
                                } else {
                                    const float kk = GAUSS ? P.cn * P.cn * 2.50662827463100050242f : P.cn * P.cn;
                                    acc[c][k].r = fmaf(amp, kk, acc[c][k].r);
                                }
                                ++evals;
                            }
                        }
                    }
                }
            }
            // ScalePressure fused with the store into [field][isz][iz][ir]
            if(have_d) {
#pragma unroll
                for(int k = 0; k < NFP; ++k) {
                    if(k >= nf) break;
                    float2 *row = out + G.field_base + (int64_t)(f0 + k) * G.field_stride_f +
                                  ((int64_t)isz * nz + d) * e.nrr + ir0;
#pragma unroll
                    for(int c = 0; c < TILE_COLS; ++c) {
                        if(c >= ncols) break;
                        float ur = acc[c][k].r, ui = acc[c][k].i;
                        if(!COHERENT) { ur = sqrtf(ur); ui = 0.f; }
                        double factor;
                        const double r = e.rr[ir0 + c];
                        if(e.line_source) factor = (double)(-4.0f * sqrtf(3.14159265f)) * FLTD(-1.0);
                        else if(fabs(r) < DBL_EPS) factor = 0.0;
                        else factor = FLTD(-1.0) / sqrt(fabs(r));
                        const float ff = (float)factor;
                        row[c] = make_float2(ur * ff, ui * ff);
                    }
                }
            }
        }
    }
    for(int o = 16; o > 0; o >>= 1) evals += __shfl_xor_sync(0xffffffffu, evals, o);
    if(lane == 0 && evals) atomicAdd(&ctr->nevals, (unsigned long long)evals);
}

template<int NFP> cudaError_t launch_tiles_nf(const void *segs, const GroupDev *groups, int ngroups,
                                              const TileGroupDev *tg, const double *freqs, const unsigned int *list,
                                              const unsigned int *off, const unsigned int *order,
                                              unsigned long long ntiles, int ndb_max, unsigned long long list_cap,
                                              float2 *out, RunCounters *ctr, bool gauss, bool coherent, int grid,
                                              cudaStream_t st)
{
    const SegRec<float> *s = (const SegRec<float> *)segs;
    const int smem = (int)(PB * sizeof(TilePrep<NFP>));
#define BHCB_TILE_LAUNCH(G_, C_)                                                                                 \
    do {                                                                                                         \
        cudaError_t e_ = cudaFuncSetAttribute(tile_kernel<NFP, G_, C_>,                                          \
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, smem);                \
        if(e_ != cudaSuccess) return e_;                                                                         \
        tile_kernel<NFP, G_, C_><<<grid, TILE_DEPTHS, smem, st>>>(s, groups, ngroups, tg, freqs, list, off, order, \
                                                                    ntiles, ndb_max, list_cap, out, ctr);        \
    } while(0)
    if(gauss && coherent) BHCB_TILE_LAUNCH(true, true);
    else if(gauss) BHCB_TILE_LAUNCH(true, false);
    else if(coherent) BHCB_TILE_LAUNCH(false, true);
    else BHCB_TILE_LAUNCH(false, false);
#undef BHCB_TILE_LAUNCH
    return cudaGetLastError();
}

} // namespace

// Bins, scan and fill of the launch's bins [b0, b1) (indexed absolutely in
// cnt, work and off; cnt and work must be zero); the tile order lists the
// launch's (bin, depth block) tiles only.
cudaError_t launch_tile_binning(const void *segs, unsigned long long cap, const RunCounters *ctr_ro,
                                RunCounters *ctr, const GroupDev *groups, int ngroups, const TileGroupDev *tg,
                                unsigned int *cnt, float *work, unsigned int *off, unsigned int *order,
                                long long b0, long long b1, int ndb_max, unsigned int *list,
                                unsigned long long list_cap, int sm_count, cudaStream_t st)
{
    const SegRec<float> *s = (const SegRec<float> *)segs;
    const int grid = sm_count * 8;
    tile_bin_kernel<false><<<grid, 256, 0, st>>>(s, cap, ctr_ro, groups, ngroups, tg, cnt, work, nullptr, 0);
    tile_scan_kernel<<<1, SCAN_THREADS, 0, st>>>(cnt + b0, off + b0, work + b0, b0, b1 - b0, ndb_max, order,
                                                 list_cap, ctr);
    tile_bin_kernel<true><<<grid, 256, 0, st>>>(s, cap, ctr_ro, groups, ngroups, tg, cnt, nullptr, list, list_cap);
    return cudaGetLastError();
}

// Resident tile CTAs per SM of the variant a launch uses.
int tile_ctas_per_sm(int nfreq_max, bool gauss, bool coherent)
{
    int n = 0;
    const void *fn;
    if(nfreq_max <= 1)
        fn = gauss ? (coherent ? (const void *)tile_kernel<1, true, true> : (const void *)tile_kernel<1, true, false>)
                   : (coherent ? (const void *)tile_kernel<1, false, true> : (const void *)tile_kernel<1, false, false>);
    else if(nfreq_max <= 4)
        fn = gauss ? (coherent ? (const void *)tile_kernel<4, true, true> : (const void *)tile_kernel<4, true, false>)
                   : (coherent ? (const void *)tile_kernel<4, false, true> : (const void *)tile_kernel<4, false, false>);
    else
        fn = gauss ? (coherent ? (const void *)tile_kernel<NFP_MAX, true, true>
                               : (const void *)tile_kernel<NFP_MAX, true, false>)
                   : (coherent ? (const void *)tile_kernel<NFP_MAX, false, true>
                               : (const void *)tile_kernel<NFP_MAX, false, false>);
    const size_t smem = PB * (nfreq_max <= 1 ? sizeof(TilePrep<1>) : nfreq_max <= 4 ? sizeof(TilePrep<4>)
                                                                                      : sizeof(TilePrep<NFP_MAX>));
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, TILE_DEPTHS, smem) != cudaSuccess || n < 1) {
        cudaGetLastError();
        n = 1;
    }
    return n;
}

cudaError_t launch_tiles(const void *segs, const GroupDev *groups, int ngroups, const TileGroupDev *tg,
                         const double *freqs, const unsigned int *list, const unsigned int *off,
                         const unsigned int *order, unsigned long long ntiles, int ndb_max, int nfreq_max,
                         unsigned long long list_cap, float2 *out, RunCounters *ctr, bool gauss, bool coherent,
                         int grid, cudaStream_t st)
{
    if(nfreq_max <= 1)
        return launch_tiles_nf<1>(segs, groups, ngroups, tg, freqs, list, off, order, ntiles, ndb_max, list_cap, out, ctr,
                                  gauss, coherent, grid, st);
    if(nfreq_max <= 4)
        return launch_tiles_nf<4>(segs, groups, ngroups, tg, freqs, list, off, order, ntiles, ndb_max, list_cap, out, ctr,
                                  gauss, coherent, grid, st);
    return launch_tiles_nf<NFP_MAX>(segs, groups, ngroups, tg, freqs, list, off, order, ntiles, ndb_max, list_cap,
                                    out, ctr, gauss, coherent, grid, st);
}

} // namespace bhcb
