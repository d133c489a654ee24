// Arrivals and eigenray hits for the 2-D field modes (RunType 'A' / 'a' / 'E').
//
// The reference adds arrivals one contribution at a time (AddArr,
// src/arrivals.hpp:45-132): a contribution either merges into the receiver's
// last arrival (when its delay and phase are within 0.05 rad of it) or is
// appended / replaces the weakest one. The result depends on the order in
// which contributions reach a receiver, and the reference's single-threaded
// order (ray by ray in job order, step by step) is the one with merging
// enabled (src/mode/arr.hpp:78). Eigen hits (RecordEigenHit,
// src/eigenrays.hpp:24-40) are likewise listed in that order.
//
// On the GPU, with all rays traced concurrently, the order is rebuilt:
//   1. arr_gather_kernel (count pass): counts the contributions;
//   2. arr_gather_kernel (fill pass): writes one candidate per contribution
//      with a 64-bit key (receiver cell, ray, step) for arrivals or (field,
//      ray, step, column walk position, depth) for eigen hits;
//   3. a stable LSD radix sort of the keys (8-bit digits; per-tile histograms,
//      one exclusive scan, warp-stable scatter);
//   4. arr_replay_kernel: one thread per receiver cell applies the AddArr rule
//      to its candidates in sorted order, then PostProcessArrivals' amplitude
//      scaling (src/mode/arr.cpp:24-74); eigen_emit_kernel writes the hits in
//      sorted order.
// The contribution math (InfluenceGeoCore, src/influence.hpp:897-1024) is FP64
// with the reference's operation order in both precisions of the tracer.
#include <cuda_runtime.h>

#include <utility>

#include "bhcb_internal.h"
#include "device_math.cuh"
#include "trace2d.cuh"
#include "influence2d.cuh"
#include "trace3d.cuh"

namespace bhcb {

namespace {

constexpr double RAD_DEG = 180.0 / BHCB_PI;
constexpr int SORT_TILE = 4096;   // keys per scatter tile (one warp)

__device__ __forceinline__ int group_of_cell(const GroupDev *groups, int ngroups, long long cell)
{
    int lo = 0, hi = ngroups - 1;
    while(lo < hi) {
        int m = (lo + hi + 1) >> 1;
        if(groups[m].field_base <= cell) lo = m; else hi = m - 1;
    }
    return lo;
}

// Walks every contribution of every segment; one thread per segment.
// COUNT: only counts (ctr->nevals). Otherwise writes candidate i with key /
// value (i) at i = atomicAdd(cursor).
template<typename R, bool GAUSS, bool COUNT>
__global__ void __launch_bounds__(128) arr_gather_kernel(
    const SegRec<R> *__restrict__ segs, unsigned long long cap, const GroupDev *__restrict__ groups,
    int ngroups, const double *__restrict__ freqs, ArrCand *cands, uint64_t *keys, uint32_t *vals,
    unsigned long long cand_cap, unsigned long long *cursor, RunCounters *ctr, ArrKeyBits kb)
{
    const unsigned long long nseg = min(__ldcg(&ctr->nseg), cap);
    unsigned long long count = 0;
    for(unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < nseg;
        k += (unsigned long long)gridDim.x * blockDim.x) {
        const SegRec<R> S = segs[k];
        if(S.job < 0) continue;
        const int gi = find_group(groups, ngroups, S.job);
        const GroupDev &G = groups[gi];
        const EnvDev &e = *G.env;
        const int local = (int)((long long)S.job - G.job_base);
        const int nal = e.isingle > 0 ? 1 : e.nalpha;
        const int isz = local / nal;
        const double freq = freqs[G.freq_base];
        // AdjustSigma (src/influence.hpp:91-100) and the depth window
        // (src/influence.hpp:1285-1292), as in the TL kernels
        R sig = S.sigma_seg, sigfloor = (R)0;
        if(GAUSS) {
            R lam = S.c0 / (R)freq;
            R fl = min((R)FLTD(0.2) * (R)freq * S.tau1r, (R)BHCB_PI * lam);
            sigfloor = fl;
            sig = max(sig, fl);
        }
        const double rmax = (GAUSS ? 4.0 : 1.0) * (double)sig;
        double zmin = -1.7976931348623157e308, zmax = 1.7976931348623157e308;
        if(fabs((double)S.tx) > FLTD(0.50001)) {
            zmin = (double)S.zlo - rmax;
            zmax = (double)S.zhi + rmax;
        }
        const bool irregular = e.irregular != 0;
        const int nrzp = e.nrz_per_range;
        int izlo = 0, izhi = 1;
        if(!irregular) {
            izlo = lower_f(e.rz, e.nrz, zmin);
            izhi = upper_f(e.rz, e.nrz, zmax);
        }
        const double tx = (double)S.tx, tz = (double)S.tz, rlen = (double)S.rlen;
        const double q0 = (double)S.q0, dq = (double)S.dq, rcpq = (double)S.rcp_q0;
        for(int ir = S.ir_lo; ir <= S.ir_hi; ++ir) {
            const double dr = e.rr[ir] - S.x0r;
            for(int iz = izlo; iz < izhi; ++iz) {
                const float zrf = irregular ? e.rz[ir] : e.rz[iz];
                if(irregular && ((double)zrf < zmin || (double)zrf > zmax)) continue;
                // InfluenceGeoCore (src/influence.hpp:897-1024), 2-D
                const double dz = (double)zrf - S.x0z;
                const double s = (dr * tx + dz * tz) / rlen;
                const double n1 = fabs(dz * tx - dr * tz);
                const double qF = q0 + s * dq;
                double sigma = fabs(qF * rcpq);
                const double sig0 = sigma;
                if(GAUSS) sigma = max(sigma, (double)sigfloor);
                if(n1 >= (GAUSS ? 4.0 : 1.0) * sigma) continue;
                if(COUNT) {
                    ++count;
                    continue;
                }
                const unsigned long long i = atomicAdd(cursor, 1ull);
                if(i >= cand_cap) continue;
                const int ialpha = e.isingle > 0 ? e.isingle - 1 : local % nal;
                uint64_t key;
                ArrCand c;
                if(kb.eigen) {
                    const int walk = S.tx > (R)0 ? ir : e.nrr - 1 - ir;
                    const int fidx = G.field_index;
                    key = ((uint64_t)fidx << kb.sh_cell) | ((uint64_t)local << kb.sh_job)
                          | ((uint64_t)S.is << kb.sh_is) | ((uint64_t)walk << kb.sh_walk) | (uint64_t)iz;
                    c.amp = 0.0;
                    c.phase = 0.0;
                    c.delay_re = 0.0;
                    c.delay_im = 0.0;
                    c.rcvr_decl = 0.f;
                    c.ntop = S.is;      // eigen: step index
                    c.nbot = ir;        // eigen: receiver range index
                    c.job = iz | (isz << 20);
                    c.aux = ialpha;
                } else {
                    const double cnst = (double)S.cnst_num / sqrt(fabs(qF));
                    double w;
                    if(GAUSS) w = exp(FLTD(-0.5) * (n1 / sigma) * (n1 / sigma)) * (sig0 / sigma);
                    else w = (sigma - n1) / sigma;
                    const bool caustic = (qF <= 0.0 && q0 > 0.0) || (qF >= 0.0 && q0 < 0.0);
                    const long long cell = G.field_base + ((long long)isz * nrzp + iz) * e.nrr + ir;
                    key = ((uint64_t)cell << kb.sh_cell) | ((uint64_t)local << kb.sh_job) | (uint64_t)S.is;
                    c.amp = cnst * w;
                    c.phase = (double)(caustic ? S.phase_b : S.phase_a);
                    c.delay_re = S.tau0r + s * (double)S.dtaur;
                    c.delay_im = (double)S.tau0i + s * (double)S.dtaui;
                    c.rcvr_decl = (float)S.rcvr_decl;
                    c.ntop = S.ntop;
                    c.nbot = S.nbot;
                    c.job = S.job;
                    c.aux = ialpha;
                }
                cands[i] = c;
                keys[i] = key;
                vals[i] = (uint32_t)i;
            }
        }
    }
    if(COUNT && count) atomicAdd(&ctr->nevals, count);
}

// ---------------------------------------------------------------- radix sort
// per-tile digit histogram, digit-major: hist[d * ntiles + tile]
__global__ void rs_hist_kernel(const uint64_t *__restrict__ keys, unsigned long long n, int shift,
                               uint32_t *hist, int ntiles)
{
    __shared__ uint32_t h[256];
    for(int d = threadIdx.x; d < 256; d += blockDim.x) h[d] = 0;
    __syncthreads();
    const int tile = blockIdx.x;
    const unsigned long long b = (unsigned long long)tile * SORT_TILE;
    const unsigned long long e = min(n, b + SORT_TILE);
    for(unsigned long long i = b + threadIdx.x; i < e; i += blockDim.x)
        atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
    __syncthreads();
    for(int d = threadIdx.x; d < 256; d += blockDim.x) hist[(size_t)d * ntiles + tile] = h[d];
}

// exclusive scan of len entries in one block of 1024 threads
__global__ void __launch_bounds__(1024) rs_scan_kernel(uint32_t *a, long long len)
{
    __shared__ uint32_t part[1024];
    __shared__ uint32_t carry;
    if(threadIdx.x == 0) carry = 0;
    __syncthreads();
    for(long long base = 0; base < len; base += 1024) {
        const long long i = base + threadIdx.x;
        const uint32_t v = i < len ? a[i] : 0u;
        part[threadIdx.x] = v;
        __syncthreads();
        for(int off = 1; off < 1024; off <<= 1) {   // Hillis-Steele inclusive scan
            uint32_t t = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
            __syncthreads();
            part[threadIdx.x] += t;
            __syncthreads();
        }
        if(i < len) a[i] = carry + part[threadIdx.x] - v;
        __syncthreads();
        if(threadIdx.x == 1023) carry += part[1023];
        __syncthreads();
    }
}

// stable scatter: one warp per tile, 32 keys at a time in order; lanes with the
// same digit are ranked by lane order (match_any), digit offsets in shared memory
__global__ void __launch_bounds__(32) rs_scatter_kernel(
    const uint64_t *__restrict__ kin, const uint32_t *__restrict__ vin, uint64_t *__restrict__ kout,
    uint32_t *__restrict__ vout, unsigned long long n, int shift, const uint32_t *__restrict__ hist,
    int ntiles)
{
    __shared__ uint32_t off[256];
    const int tile = blockIdx.x, lane = threadIdx.x;
    for(int d = lane; d < 256; d += 32) off[d] = hist[(size_t)d * ntiles + tile];
    __syncwarp();
    const unsigned long long b = (unsigned long long)tile * SORT_TILE;
    const unsigned long long e = min(n, b + SORT_TILE);
    for(unsigned long long i0 = b; i0 < e; i0 += 32) {
        const unsigned long long i = i0 + lane;
        const bool have = i < e;
        uint64_t k = 0;
        uint32_t v = 0;
        uint32_t d = 256u + lane;   // distinct dummy digit for idle lanes
        if(have) {
            k = kin[i];
            v = vin[i];
            d = (uint32_t)((k >> shift) & 255u);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if(have) base = off[d];
        __syncwarp();
        if(have) {
            kout[base + rank] = k;
            vout[base + rank] = v;
            if(lane == leader) off[d] = base + __popc(peers);
        }
        __syncwarp();
    }
}

// -------------------------------------------------------------- replay
// AddArr (src/arrivals.hpp:45-132) over one receiver cell's candidates in
// (ray, step) order, then PostProcessArrivals (src/mode/arr.cpp:24-74).
// D3: 3-D run (source angles from the 3-D job, receiver azimuth from the
// candidate, no amplitude scaling); the replay continues from the counts
// already in narr_out, so job-ordered waves compose.
template<bool D3>
__global__ void arr_replay_kernel(const uint64_t *__restrict__ keys, const uint32_t *__restrict__ vals,
                                  const ArrCand *__restrict__ cands, unsigned long long n,
                                  const GroupDev *__restrict__ groups, int ngroups,
                                  const double *__restrict__ freqs, long long ncells, int sh_cell,
                                  int max_narr, int allow_merging, int32_t *narr_out, ArrivalRec *arr_out)
{
    for(long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x; cell < ncells;
        cell += (long long)gridDim.x * blockDim.x) {
        // candidate range of this cell in the sorted keys
        const uint64_t klo = (uint64_t)cell << sh_cell, khi = (uint64_t)(cell + 1) << sh_cell;
        unsigned long long lo = 0, hi = n;
        while(lo < hi) {
            unsigned long long m = (lo + hi) >> 1;
            if(keys[m] < klo) lo = m + 1; else hi = m;
        }
        const unsigned long long begin = lo;
        hi = n;
        while(lo < hi) {
            unsigned long long m = (lo + hi) >> 1;
            if(keys[m] < khi) lo = m + 1; else hi = m;
        }
        const unsigned long long end = lo;
        const GroupDev &G = groups[group_of_cell(groups, ngroups, cell)];
        const double omega = D3 ? 2.0 * BHCB_PI * G.env3->freq0 : 2.0 * BHCB_PI * freqs[G.freq_base];
        ArrivalRec *ba = arr_out + (size_t)cell * max_narr;
        int nt = D3 ? narr_out[cell] : 0;
        for(unsigned long long k = begin; k < end; ++k) {
            const ArrCand &c = cands[vals[k]];
            double src_decl, src_azim_d = 0.0;
            float rcvr_azim;
            if(D3) {
                const Job3 J = job_indices3(*G.env3, (int)((long long)c.job - G.job_base));
                src_decl = RAD_DEG * G.env3->alpha[J.ialpha];
                src_azim_d = RAD_DEG * G.env3->beta[J.ibeta];
                rcvr_azim = c.rcvr_azim;
            } else {
                src_decl = RAD_DEG * G.env->alpha[c.aux];
                rcvr_azim = __int_as_float(0x7fc00000);   // NaN: no azimuth in 2-D
            }
            const float azim = D3 ? (float)src_azim_d : __int_as_float(0x7fc00000);
            if(allow_merging) {
                const float PhaseTol = 0.05f;
                bool second = false;
                if(nt >= 1) {
                    const ArrivalRec &L = ba[nt - 1];
                    const double ddr = c.delay_re - (double)L.delay_re, ddi = c.delay_im - (double)L.delay_im;
                    second = omega * hypot(ddr, ddi) < (double)PhaseTol
                             && fabs((double)L.Phase - c.phase) < (double)PhaseTol;
                }
                if(!second) {
                    int iArr;
                    if(nt >= max_narr) {
                        iArr = -1;
                        double weakest = c.amp;
                        for(int j = 0; j < max_narr; ++j)
                            if((double)ba[j].a < weakest) {
                                weakest = (double)ba[j].a;
                                iArr = j;
                            }
                        if(iArr < 0) continue;
                    } else {
                        iArr = nt++;
                    }
                    ArrivalRec &A = ba[iArr];
                    A.a = (float)c.amp;
                    A.Phase = (float)c.phase;
                    A.delay_re = (float)c.delay_re;
                    A.delay_im = (float)c.delay_im;
                    A.SrcDeclAngle = (float)src_decl;
                    A.SrcAzimAngle = azim;
                    A.RcvrDeclAngle = c.rcvr_decl;
                    A.RcvrAzimAngle = rcvr_azim;
                    A.NTopBnc = c.ntop;
                    A.NBotBnc = c.nbot;
                } else {
                    ArrivalRec &A = ba[nt - 1];
                    const float amp = (float)c.amp;
                    const float tot = __fadd_rn(A.a, amp);
                    const float w1 = __fdiv_rn(A.a, tot), w2 = __fdiv_rn(amp, tot);
                    A.delay_re = __fadd_rn(__fmul_rn(w1, A.delay_re), __fmul_rn(w2, (float)c.delay_re));
                    A.delay_im = __fadd_rn(__fmul_rn(w1, A.delay_im), __fmul_rn(w2, (float)c.delay_im));
                    A.a = tot;
                    A.SrcDeclAngle = __fadd_rn(__fmul_rn(w1, A.SrcDeclAngle), __fmul_rn(w2, (float)src_decl));
                    A.SrcAzimAngle = __fadd_rn(__fmul_rn(w1, A.SrcAzimAngle), __fmul_rn(w2, azim));
                    A.RcvrDeclAngle = __fadd_rn(__fmul_rn(w1, A.RcvrDeclAngle), __fmul_rn(w2, c.rcvr_decl));
                    A.RcvrAzimAngle = __fadd_rn(__fmul_rn(w1, A.RcvrAzimAngle), __fmul_rn(w2, rcvr_azim));
                }
            } else {
                const int j = nt++;
                if(j >= max_narr) continue;
                ArrivalRec &A = ba[j];
                A.a = (float)c.amp;
                A.Phase = (float)c.phase;
                A.delay_re = (float)c.delay_re;
                A.delay_im = (float)c.delay_im;
                A.SrcDeclAngle = (float)src_decl;
                A.SrcAzimAngle = azim;
                A.RcvrDeclAngle = c.rcvr_decl;
                A.RcvrAzimAngle = rcvr_azim;
                A.NTopBnc = c.ntop;
                A.NBotBnc = c.nbot;
            }
        }
        // PostProcessArrivals (src/mode/arr.cpp:24-74): clamp the count; 2-D
        // and Nx2D scale the amplitudes (3-D factor 1)
        if(nt > max_narr) nt = max_narr;
        narr_out[cell] = nt;
        if(D3 && !G.env3->nx2d) continue;
        // 2-D rays (2-D and Nx2D): cylindrical spreading per receiver range,
        // the last index of both field layouts
        const double *rr = D3 ? G.env3->rr : G.env->rr;
        const int nrr = D3 ? G.env3->nrr : G.env->nrr;
        const int ir = (int)((cell - G.field_base) % nrr);
        float factor;
        if(!D3 && G.env->line_source) factor = (float)(FLTD(4.0) * sqrt(BHCB_PI));
        else if(fabs(rr[ir]) < DBL_EPS) factor = 1e5f;
        else factor = (float)(FLTD(1.0) / sqrt(rr[ir]));
        for(int j = 0; j < nt; ++j) ba[j].a = __fmul_rn(ba[j].a, factor);
    }
}

// eigen hits in sorted order (RecordEigenHit layout, include/bhc/structs.hpp:353-361)
__global__ void eigen_emit_kernel(const uint32_t *__restrict__ vals, const ArrCand *__restrict__ cands,
                                  unsigned long long n, EigenHitRec *hits, int32_t *field_of_hit, int sh_cell,
                                  const uint64_t *__restrict__ keys)
{
    for(unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < n;
        k += (unsigned long long)gridDim.x * blockDim.x) {
        const ArrCand &c = cands[vals[k]];
        EigenHitRec h;
        h.is = c.ntop;
        h.itheta = 0;
        h.ir = c.nbot;
        h.iz = c.job & 0xfffff;
        h.isx = 0;
        h.isy = 0;
        h.isz = c.job >> 20;
        h.ialpha = c.aux;
        h.ibeta = 0;
        hits[k] = h;
        field_of_hit[k] = (int32_t)(keys[k] >> sh_cell);
    }
}

} // namespace

template<typename R> cudaError_t launch_arr_gather(const void *segs, unsigned long long cap,
                                                   const GroupDev *groups, int ngroups, const double *freqs,
                                                   bool gauss, bool count, ArrCand *cands, uint64_t *keys,
                                                   uint32_t *vals, unsigned long long cand_cap,
                                                   unsigned long long *cursor, RunCounters *ctr, ArrKeyBits kb,
                                                   int grid, cudaStream_t st)
{
    const SegRec<R> *s = (const SegRec<R> *)segs;
    if(gauss && count)
        arr_gather_kernel<R, true, true><<<grid, 128, 0, st>>>(s, cap, groups, ngroups, freqs, cands, keys, vals,
                                                               cand_cap, cursor, ctr, kb);
    else if(gauss)
        arr_gather_kernel<R, true, false><<<grid, 128, 0, st>>>(s, cap, groups, ngroups, freqs, cands, keys, vals,
                                                                cand_cap, cursor, ctr, kb);
    else if(count)
        arr_gather_kernel<R, false, true><<<grid, 128, 0, st>>>(s, cap, groups, ngroups, freqs, cands, keys, vals,
                                                                cand_cap, cursor, ctr, kb);
    else
        arr_gather_kernel<R, false, false><<<grid, 128, 0, st>>>(s, cap, groups, ngroups, freqs, cands, keys,
                                                                 vals, cand_cap, cursor, ctr, kb);
    return cudaGetLastError();
}
template cudaError_t launch_arr_gather<float>(const void *, unsigned long long, const GroupDev *, int,
                                              const double *, bool, bool, ArrCand *, uint64_t *, uint32_t *,
                                              unsigned long long, unsigned long long *, RunCounters *, ArrKeyBits,
                                              int, cudaStream_t);
template cudaError_t launch_arr_gather<double>(const void *, unsigned long long, const GroupDev *, int,
                                               const double *, bool, bool, ArrCand *, uint64_t *, uint32_t *,
                                               unsigned long long, unsigned long long *, RunCounters *, ArrKeyBits,
                                               int, cudaStream_t);

size_t radix_sort_hist_entries(unsigned long long n)
{
    return (size_t)256 * (size_t)((n + SORT_TILE - 1) / SORT_TILE);
}

// Sorts (keys, vals) by the low `bits` bits of the keys; the result is in
// (k0, v0) when the number of passes is even, else in (k1, v1): returns which.
cudaError_t radix_sort_pairs(uint64_t *k0, uint32_t *v0, uint64_t *k1, uint32_t *v1, unsigned long long n,
                             int bits, uint32_t *hist, int *result_in_1, cudaStream_t st)
{
    *result_in_1 = 0;
    if(n == 0) return cudaSuccess;
    const int ntiles = (int)((n + SORT_TILE - 1) / SORT_TILE);
    uint64_t *ki = k0, *ko = k1;
    uint32_t *vi = v0, *vo = v1;
    int passes = 0;
    for(int shift = 0; shift < bits; shift += 8, ++passes) {
        rs_hist_kernel<<<ntiles, 256, 0, st>>>(ki, n, shift, hist, ntiles);
        rs_scan_kernel<<<1, 1024, 0, st>>>(hist, (long long)256 * ntiles);
        rs_scatter_kernel<<<ntiles, 32, 0, st>>>(ki, vi, ko, vo, n, shift, hist, ntiles);
        std::swap(ki, ko);
        std::swap(vi, vo);
    }
    *result_in_1 = passes & 1;
    return cudaGetLastError();
}

cudaError_t launch_arr_replay(const uint64_t *keys, const uint32_t *vals, const ArrCand *cands, unsigned long long n,
                              const GroupDev *groups, int ngroups, const double *freqs, long long ncells, int sh_cell,
                              int max_narr, int allow_merging, int32_t *narr, ArrivalRec *arr, int sm_count,
                              cudaStream_t st, bool d3)
{
    long long grid = (ncells + 127) / 128;
    if(grid > (long long)sm_count * 64) grid = (long long)sm_count * 64;
    if(grid < 1) grid = 1;
    if(d3)
        arr_replay_kernel<true><<<(int)grid, 128, 0, st>>>(keys, vals, cands, n, groups, ngroups, freqs, ncells,
                                                           sh_cell, max_narr, allow_merging, narr, arr);
    else
        arr_replay_kernel<false><<<(int)grid, 128, 0, st>>>(keys, vals, cands, n, groups, ngroups, freqs, ncells,
                                                            sh_cell, max_narr, allow_merging, narr, arr);
    return cudaGetLastError();
}

cudaError_t launch_eigen_emit(const uint32_t *vals, const ArrCand *cands, unsigned long long n, EigenHitRec *hits,
                              int32_t *field_of_hit, int sh_cell, const uint64_t *keys, int sm_count, cudaStream_t st)
{
    long long grid = (long long)((n + 255) / 256);
    if(grid > (long long)sm_count * 32) grid = (long long)sm_count * 32;
    if(grid < 1) grid = 1;
    eigen_emit_kernel<<<(int)grid, 256, 0, st>>>(vals, cands, n, hits, field_of_hit, sh_cell, keys);
    return cudaGetLastError();
}

} // namespace bhcb
