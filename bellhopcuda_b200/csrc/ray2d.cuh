// 2-D ray driver shared by the field-mode trace kernels: segment-slot
// allocation in per-ray blocks, the per-ray state, RayInit, RayUpdate and
// RayTerminate's stop conditions (src/trace.hpp:76-477).
#pragma once
#include "bhcb_internal.h"
#include "device_math.cuh"
#include "trace2d.cuh"
#include "influence2d.cuh"

namespace bhcb {

// Segment slots are handed out to each ray in blocks of SEG_BLOCK (one global
// atomic per block); a ray's segments are therefore stored in step order.
constexpr int SEG_BLOCK = 32;

struct SlotCursor {
    unsigned long long next = 0, end = 0;   // [next, end) free slots of the current block
};

// Marks the block that ends at slot `end` as complete for the influence
// kernels that run while the trace is still going: its records are made
// visible device-wide before the flag.
__device__ __forceinline__ void publish_block(unsigned int *blk_state, unsigned long long end)
{
    if(!blk_state || end == 0) return;
    __threadfence();
    atomicExch(&blk_state[end / SEG_BLOCK - 1], 1u);
}

template<typename Rec> __device__ __forceinline__ void emit_seg(
    const Rec &rec, Rec *segs, unsigned long long cap, RunCounters *ctr, SlotCursor &cur,
    bool &overflow, unsigned int *blk_state)
{
    if(cur.next == cur.end) {
        publish_block(blk_state, cur.end);   // the previous block is full
        unsigned long long b = atomicAdd(&ctr->nseg, (unsigned long long)SEG_BLOCK);
        if(b + SEG_BLOCK > cap) {
            overflow = true;
            return;
        }
        cur.next = b;
        cur.end = b + SEG_BLOCK;
    }
    static_assert(sizeof(Rec) % 16 == 0, "segment records are written in 16-byte words");
    const uint4 *src = reinterpret_cast<const uint4 *>(&rec);
    uint4 *dst = reinterpret_cast<uint4 *>(segs + cur.next++);
#pragma unroll
    for(int k = 0; k < (int)(sizeof(Rec) / 16); ++k) dst[k] = src[k];
}

// mark the unused tail of the ray's last block as empty
template<typename Rec> __device__ __forceinline__ void close_block(Rec *segs, SlotCursor &cur,
                                                                  unsigned int *blk_state)
{
    for(; cur.next < cur.end; ++cur.next) segs[cur.next].job = -1;
    publish_block(blk_state, cur.end);
}

// Per-ray state between steps of the 2-D ray loop.
template<typename R> struct RayState2 {
    RayPt<R> p0;
    BdState top, bot;
    HsDev htop, hbot;
    SegState iSeg;
    SspSegCache sc;
    double dBegTop, dBegBot;
    double alpha;
    R c;
};

// RayInit (src/trace.hpp:76-266), 2-D: false when the source is on or outside
// the boundaries (the ray is not traced)
template<typename R> __device__ __forceinline__ bool ray_init2d(const EnvDev &e, int ialpha, int isz,
                                                                RayState2<R> &st, RunCounters *ctr)
{
    st.iSeg = SegState{0, 0};
    ssp_cache_init(st.sc, e);
    const double alpha = e.alpha[ialpha];
    st.alpha = alpha;
    const double SrcDecl = (180.0 / BHCB_PI) * alpha;
    const V2<double> xs = mk2(0.0, (double)e.sz[isz]);
    const V2<R> tinit = mk2((R)e.acs[2 * ialpha], (R)e.acs[2 * ialpha + 1]);
    SSPOut<R> o;
    eval_ssp(xs, tinit, o, e, st.iSeg, ctr);
    const R c = o.c;
    st.c = c;
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
    RayPt<R> &p0 = st.p0;
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
    st.htop = e.top;
    st.hbot = e.bot;
    st.top.Iseg = st.bot.Iseg = 0;
    st.top.lmin = st.top.lmax = st.bot.lmin = st.bot.lmax = 0.0;
    get_bdry_seg(xs, (double)p0.t.x, st.top, e.btop, e.ntop, e.top_long, st.htop, true, true, ctr);
    get_bdry_seg(xs, (double)p0.t.x, st.bot, e.bbot, e.nbot, e.bot_long, st.hbot, false, true, ctr);
    distances(xs, st.top, st.bot, st.dBegTop, st.dBegBot);
    if(st.dBegTop <= 0.0 || st.dBegBot <= 0.0) {
        run_warn(ctr, WARN_SOURCE_OUTSIDE_BOUNDARIES);
        return false;
    }
    return true;
}

// RayUpdate (src/trace.hpp:274-381), 2-D: one step from st.p0 to p1 and, on a
// boundary hit, the reflected point p2; returns whether p2 was produced
template<typename R> __device__ __forceinline__ bool ray_update2d(RayState2<R> &st, RayPt<R> &p1, RayPt<R> &p2,
                                                                  int &small, double &dEndTop, double &dEndBot,
                                                                  const EnvDev &e, RunCounters *ctr)
{
    bool tr = false, br = false;
    step2d(st.p0, p1, st.top, st.bot, e, st.iSeg, small, tr, br, ctr, &st.sc);
    get_bdry_seg(p1.x, (double)p1.t.x, st.top, e.btop, e.ntop, e.top_long, st.htop, true, false, ctr);
    get_bdry_seg(p1.x, (double)p1.t.x, st.bot, e.bbot, e.nbot, e.bot_long, st.hbot, false, false, ctr);
    distances(p1.x, st.top, st.bot, dEndTop, dEndBot);
    const bool two = tr || br;
    if(two) {
        const BdryPtDev *bd = tr ? e.btop : e.bbot;
        const BdState &bs = tr ? st.top : st.bot;
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
        reflect2d(p1, p2, tr ? st.htop : st.hbot, tr, tI, nI, (R)b0.kappa, e, st.iSeg, ctr);
        distances(p2.x, st.top, st.bot, dEndTop, dEndBot);
    }
    return two;
}

// RayTerminate's stop conditions (src/trace.hpp:391-477), 2-D
template<typename R> __device__ __forceinline__ bool ray_stops2d(const RayState2<R> &st, double dEndTop,
                                                                 double dEndBot, const EnvDev &e)
{
    const RayPt<R> &p0 = st.p0;
    const bool leftbox = fabs(p0.x.x) >= e.box_x || fabs(p0.x.y) >= e.box_y;
    const bool escaped = (st.dBegTop < 0.0 && dEndTop < 0.0) || (st.dBegBot < 0.0 && dEndBot < 0.0);
    const bool lost = (double)p0.Amp < FLTD(0.005);
    return leftbox || lost || escaped;
}

} // namespace bhcb
