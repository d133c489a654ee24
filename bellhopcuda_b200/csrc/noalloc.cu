// bhcb_run_noalloc: one TL field into a caller-owned device buffer without any
// device (or host) memory allocation during the call.
//
// Who needs this: callers that must not allocate once they are running — code
// that works inside a fixed device-memory budget owned by another allocator
// (a framework's caching allocator that holds the free memory), real-time
// loops with an allocation-free policy after initialisation. They prepare a
// context once (bhcb_open / bhcb_setup / bhcb_prepare, which do allocate),
// then call this entry point as often as they like. The call is synchronous
// (it copies the run header in and the counters out and waits for the
// context stream); work that is to be captured into a CUDA graph uses the
// bhcb_graph_* entry points below instead.
//
// How: it runs a variant of the trace kernel that evaluates each segment's
// beam-receiver contributions inline instead of storing segment records, so
// the only scratch it needs is the range-major accumulator, the run counters
// and the one-field scale descriptor. Those live in g_noalloc_scratch, a
// file-scope __device__ array of 256 B + 8 B x BHCB_NOALLOC_MAX_FIELD
// (16 MiB + 256 B) that every GPU which loads the library holds until the
// process exits. Host code cannot use the
// array's name as a device address, so the first call on each device, with
// that device (the context's GPU) made current, looks the address up with
// cudaGetSymbolAddress and keeps it. Every call runs on the context's GPU and
// restores the caller's current device before it returns.
//
// All calls on a device share the array: each call clears the counters and
// the accumulator before use, and two calls whose GPU work overlaps (two
// streams, two threads) race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/bhcb.h"
#include "bhcb_internal.h"
#include "device_math.cuh"
#include "influence2d.cuh"
#include "noalloc.h"
#include "trace2d.cuh"

namespace bhcb {

cudaError_t launch_scale(const float2 *, float2 *, const GroupDev *, int, int, cudaStream_t);

namespace {

struct NoAllocHeader {
    RunCounters ctr;
    unsigned long long job_counter;
    GroupDev group;   // the scale kernel reads the field descriptor from device memory
};
static_assert(sizeof(NoAllocHeader) <= 256, "header must fit in the first 256 bytes");

constexpr size_t kHeaderBytes = 256;
constexpr size_t kAccBytes = (size_t)BHCB_NOALLOC_MAX_FIELD * sizeof(float2);

__device__ __align__(256) static unsigned char g_noalloc_scratch[kHeaderBytes + kAccBytes];

constexpr int kMaxDevices = 64;
void *g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

// Contributions of one segment for one frequency, evaluated by the thread
// that traced it (InfluenceGeoCore + ApplyContribution,
// src/influence.hpp:423-473,897-1024, 2-D Cartesian).
template<typename R, bool GAUSS, bool COHERENT> __device__ __forceinline__ void eval_segment_inline(
    const SegRec<R> &S, const EnvDev &e, double freq, float2 *acc, long long base,
    unsigned long long &evals)
{
    using M = EvalMath<R>;
    double omega = 2.0 * BHCB_PI * freq;
    R sig = S.sigma_seg, sigfloor = (R)0;
    if(GAUSS) {   // AdjustSigma (src/influence.hpp:91-100)
        R lam = S.c0 / (R)freq;
        sigfloor = min((R)FLTD(0.2) * (R)freq * S.tau1r, (R)BHCB_PI * lam);
        sig = max(sig, sigfloor);
    }
    double rmax = (GAUSS ? 4.0 : 1.0) * (double)sig;
    double zmin = -1.7976931348623157e308, zmax = 1.7976931348623157e308;
    if(fabs((double)S.tx) > FLTD(0.50001)) {   // steep segments take every depth
        zmin = (double)S.zlo - rmax;
        zmax = (double)S.zhi + rmax;
    }
    int izlo = 0, niz = e.nrz;
    if(e.irregular) {
        niz = 1;
    } else {
        izlo = lower_f(e.rz, e.nrz, zmin);
        niz = upper_f(e.rz, e.nrz, zmax) - izlo;
    }
    R ph0 = (R)reduce_2pi(omega * S.tau0r);
    R omdt = (R)(omega * (double)S.dtaur);
    R att0 = (R)(omega * (double)S.tau0i), att1 = (R)(omega * (double)S.dtaui);
    int nrzp = e.irregular ? 0 : e.nrz_per_range;
    for(int ir = S.ir_lo; ir <= S.ir_hi; ++ir) {
        for(int j = 0; j < niz; ++j) {
            int iz = izlo + j;
            double zr = (double)e.rz[nrzp ? iz : ir];
            if(!nrzp && (zr < zmin || zr > zmax)) continue;   // depth window, irregular grid
            R dr = (R)(e.rr[ir] - S.x0r), dz = (R)(zr - S.x0z);
            R s = M::div(dr * S.tx + dz * S.tz, S.rlen);
            R n1 = fabs(dz * S.tx - dr * S.tz);
            R qF = S.q0 + s * S.dq;
            R sigma = fabs(qF * S.rcp_q0);
            R sig0 = sigma;
            if(GAUSS) sigma = max(sigma, sigfloor);
            if(n1 >= (GAUSS ? (R)4 : (R)1) * sigma) continue;
            R cnst = S.cnst_num * M::rsqrt_(fabs(qF));
            R wgt;
            if(GAUSS) {
                R a = M::div(n1, sigma);
                wgt = M::exp_((R)FLTD(-0.5) * a * a) * M::div(sig0, sigma);
            } else {
                wgt = M::div(sigma - n1, sigma);
            }
            bool caustic = (qF <= (R)0 && S.q0 > (R)0) || (qF >= (R)0 && S.q0 < (R)0);
            R ph = caustic ? S.phase_b : S.phase_a;
            float2 v;
            if(COHERENT) {
                R amp = cnst * wgt * M::exp_(att0 + s * att1);
                R ang = reduce_2pi(ph0 + s * omdt - ph);
                R sn, cs;
                M::sincos_(ang, &sn, &cs);
                v = make_float2((float)(amp * cs), (float)(-amp * sn));
            } else {
                R vv = cnst * M::exp_(att0 + s * att1);
                vv = vv * vv * wgt;
                if(GAUSS) vv *= (R)sqrt(FLTD(2.0) * BHCB_PI);
                v = make_float2((float)vv, 0.f);
            }
            atomicAdd(&acc[base + (long long)ir * (nrzp ? nrzp : 1) + (nrzp ? iz : 0)], v);
            ++evals;
        }
    }
}

// Variant of trace_kernel (kernels2d.cu) for one trace group and one
// frequency: same ray physics (src/trace.hpp:76-589), contributions applied
// inline into the static accumulator.
template<typename R, typename RecR, bool GAUSS, bool COHERENT> __global__ void __launch_bounds__(64)
noalloc_trace_kernel(unsigned char *scratch, double freq)
{
    NoAllocHeader *H = reinterpret_cast<NoAllocHeader *>(scratch);
    float2 *acc = reinterpret_cast<float2 *>(scratch + kHeaderBytes);
    RunCounters *ctr = &H->ctr;
    const GroupDev G = H->group;
    const EnvDev &e = *G.env;
    unsigned long long evals = 0;
    for(;;) {
        long long job = (long long)atomicAdd(&H->job_counter, 1ull);
        if(job >= G.njobs) break;
        int nalpha_eff = e.isingle > 0 ? 1 : e.nalpha;
        int ialpha = e.isingle > 0 ? e.isingle - 1 : (int)job % nalpha_eff;
        int isz = (int)job / nalpha_eff;
        if(isz >= e.nsz) { run_error(ctr, ERR_RAYINIT); continue; }
        long long base = (long long)isz * e.nrr * e.nrz_per_range;

        SegState iSeg{0, 0};
        double alpha = e.alpha[ialpha];
        double SrcDecl = (180.0 / BHCB_PI) * alpha;
        V2<double> xs = mk2(0.0, (double)e.sz[isz]);
        V2<R> tinit = mk2((R)e.acs[2 * ialpha], (R)e.acs[2 * ialpha + 1]);
        SSPOut<R> o;
        eval_ssp(xs, tinit, o, e, iSeg, ctr);
        R c = o.c;
        int ibp = min(bsearch_leq2(e.sbp, e.nsbp, SrcDecl), e.nsbp - 2);
        double sb = (SrcDecl - e.sbp[2 * ibp]) / (e.sbp[2 * (ibp + 1)] - e.sbp[2 * ibp]);
        float amp0 = (float)((FLTD(1.0) - sb) * e.sbp[2 * ibp + 1] + sb * e.sbp[2 * (ibp + 1) + 1]);
        if(e.run0 == 'S') {
            float om = (float)(FLTD(2.0) * BHCB_PI * freq);
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
        unsigned long long nsteps = 0;
        for(;;) {
            if((nsteps & 31) == 0 && __ldcg(&ctr->err_bits) != 0u) break;
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
            SegRec<RecR> rec;
            if(infl_prologue(p0, p1, inf, e, rcp_q0, ratio1, (int)job, is, rec))
                eval_segment_inline<RecR, GAUSS, COHERENT>(rec, e, freq, acc, base, evals);
            ++is;
            if(two) {
                if(infl_prologue(p1, p2, inf, e, rcp_q0, ratio1, (int)job, is, rec))
                    eval_segment_inline<RecR, GAUSS, COHERENT>(rec, e, freq, acc, base, evals);
                p0 = p2;
                ++is;
            } else {
                p0 = p1;
            }
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
    if(evals) atomicAdd(&ctr->nevals, evals);
}

// R: contribution precision; the ray state is FP64 in both precisions, as in
// the trace kernel
template<typename R> void launch_fused(const NoAllocJob &J, unsigned char *scratch, int grid)
{
    if(J.gaussian && J.coherent)
        noalloc_trace_kernel<double, R, true, true><<<grid, 32, 0, J.stream>>>(scratch, J.freq);
    else if(J.gaussian)
        noalloc_trace_kernel<double, R, true, false><<<grid, 32, 0, J.stream>>>(scratch, J.freq);
    else if(J.coherent)
        noalloc_trace_kernel<double, R, false, true><<<grid, 32, 0, J.stream>>>(scratch, J.freq);
    else
        noalloc_trace_kernel<double, R, false, false><<<grid, 32, 0, J.stream>>>(scratch, J.freq);
}

// Makes the context's GPU current for the lifetime of the guard and gives the
// caller's current device back afterwards.
struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    explicit DeviceGuard(int dev)
    {
        if(cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard()
    {
        if(prev >= 0) cudaSetDevice(prev);
    }
};

int put_msg(char *msg, size_t n, int code, const char *text)
{
    if(msg && n) {
        size_t l = strlen(text);
        if(l > n - 1) l = n - 1;
        memcpy(msg, text, l);
        msg[l] = 0;
    }
    return code;
}

} // namespace
} // namespace bhcb

using namespace bhcb;

extern "C" int bhcb_run_noalloc(bhcb_ctx *ctx, int32_t env_index, int32_t ifreq, void *field_dev,
                                size_t bytes, char *msg, size_t msg_len)
{
    if(msg && msg_len) msg[0] = 0;
    if(!ctx || !field_dev) return put_msg(msg, msg_len, BHCB_ERR_ARG, "context or output pointer is NULL");
    NoAllocJob J;
    const char *why = nullptr;
    int rc = noalloc_job_from_ctx(ctx, env_index, ifreq, &J, &why);
    if(rc != BHCB_OK) return put_msg(msg, msg_len, rc, why ? why : "invalid request");
    size_t nelem = (size_t)J.nsz * J.nrzp * J.nrr;
    if(nelem > (size_t)BHCB_NOALLOC_MAX_FIELD) {
        char b[160];
        snprintf(b, sizeof b, "field of %zu receivers exceeds the static scratch limit of %d receivers "
                 "(BHCB_NOALLOC_MAX_FIELD); use bhcb_run", nelem, (int)BHCB_NOALLOC_MAX_FIELD);
        return put_msg(msg, msg_len, BHCB_ERR_ARG, b);
    }
    if(bytes < nelem * sizeof(float2)) return put_msg(msg, msg_len, BHCB_ERR_ARG, "output buffer too small");
    const int dev = J.device;
    if(dev < 0 || dev >= kMaxDevices) return put_msg(msg, msg_len, BHCB_ERR_CUDA, "context device out of range");
    // the context's stream, tables and the caller's buffer live on the
    // context's GPU: run there whatever device the caller has current
    DeviceGuard guard(dev);
    if(!guard.ok) return put_msg(msg, msg_len, BHCB_ERR_CUDA, "cannot make the context's device current");
    void *scratch = nullptr;
    {
        // one-time set-up per device, with that device current
        std::lock_guard<std::mutex> lk(g_scratch_mutex);
        if(!g_scratch_addr[dev]) {
            void *p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if(e != cudaSuccess || !p)
                return put_msg(msg, msg_len, BHCB_ERR_CUDA, "cudaGetSymbolAddress of the static scratch failed");
            g_scratch_addr[dev] = p;
        }
        scratch = g_scratch_addr[dev];
    }
    // header: zeroed counters, job counter, and the field descriptor of this
    // single field written at offset 0 of the accumulator / output
    NoAllocHeader h;
    memset(&h, 0, sizeof h);
    h.ctr.overflow_job = 0xffffffffu;
    h.group = J.group;
    h.group.job_base = 0;
    h.group.nfreq = 1;
    h.group.freq_base = 0;
    h.group.field_base = 0;
    h.group.field_stride_f = (int)nelem;
    h.group.acc_base = 0;                  // this path's accumulator rows are not padded
    h.group.acc_stride_f = (int64_t)nelem;
    h.group.acc_nz = J.nrzp;
    unsigned char *sc = (unsigned char *)scratch;
    if(cudaMemcpyAsync(sc, &h, sizeof h, cudaMemcpyHostToDevice, J.stream) != cudaSuccess
       || cudaMemsetAsync(sc + kHeaderBytes, 0, nelem * sizeof(float2), J.stream) != cudaSuccess)
        return put_msg(msg, msg_len, BHCB_ERR_CUDA, "clearing the static scratch failed");
    long long grid = (J.group.njobs + 31) / 32;
    if(grid > (long long)J.sm_count * 16) grid = (long long)J.sm_count * 16;
    if(grid < 1) grid = 1;
    if(J.precision == BHCB_PREC_FP64) launch_fused<double>(J, sc, (int)grid);
    else launch_fused<float>(J, sc, (int)grid);
    if(cudaGetLastError() != cudaSuccess)
        return put_msg(msg, msg_len, BHCB_ERR_CUDA, "kernel launch failed");
    NoAllocHeader *dh = reinterpret_cast<NoAllocHeader *>(sc);
    if(launch_scale(reinterpret_cast<const float2 *>(sc + kHeaderBytes), (float2 *)field_dev, &dh->group, 1,
                    J.sm_count * 2, J.stream) != cudaSuccess)
        return put_msg(msg, msg_len, BHCB_ERR_CUDA, "scale launch failed");
    RunCounters back;
    if(cudaMemcpyAsync(&back, &dh->ctr, sizeof back, cudaMemcpyDeviceToHost, J.stream) != cudaSuccess
       || cudaStreamSynchronize(J.stream) != cudaSuccess)
        return put_msg(msg, msg_len, BHCB_ERR_CUDA, "synchronising the run failed");
    if(back.err_bits) {
        char b[96];
        snprintf(b, sizeof b, "tracer error bits 0x%x", back.err_bits);
        return put_msg(msg, msg_len, BHCB_ERR_RUN, b);
    }
    return BHCB_OK;
}

// ------------------------------------------------------------ CUDA graphs
// A prepared field captured once into a CUDA graph (header set-up, accumulator
// clear, fused trace + influence, scale) and replayed with one
// cudaGraphLaunch per run. The graph owns its scratch (allocated before the
// capture), so graphs of different fields can be replayed concurrently.
struct bhcb_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned char *scratch = nullptr;
    cudaStream_t stream = nullptr;
    int device = 0;
};

namespace bhcb {
namespace {
__global__ void write_header_kernel(NoAllocHeader h, unsigned char *dst)
{
    const unsigned *src = reinterpret_cast<const unsigned *>(&h);
    unsigned *d = reinterpret_cast<unsigned *>(dst);
    for(int i = threadIdx.x; i < (int)(sizeof(NoAllocHeader) / 4); i += blockDim.x) d[i] = src[i];
}
} // namespace
} // namespace bhcb

extern "C" void bhcb_graph_destroy(bhcb_graph *g)
{
    if(!g) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(g->device);
    if(g->stream) cudaStreamSynchronize(g->stream);
    if(g->exec) cudaGraphExecDestroy(g->exec);
    if(g->graph) cudaGraphDestroy(g->graph);
    if(g->scratch) cudaFree(g->scratch);
    if(g->stream) cudaStreamDestroy(g->stream);
    cudaSetDevice(cur);
    delete g;
}

extern "C" int bhcb_graph_create(bhcb_ctx *ctx, int32_t env_index, int32_t ifreq, void *field_dev, size_t bytes,
                                 bhcb_graph **out, char *msg, size_t msg_len)
{
    if(msg && msg_len) msg[0] = 0;
    if(!out) return put_msg(msg, msg_len, BHCB_ERR_ARG, "graph output pointer is NULL");
    *out = nullptr;
    if(!ctx || !field_dev) return put_msg(msg, msg_len, BHCB_ERR_ARG, "context or output pointer is NULL");
    NoAllocJob J;
    const char *why = nullptr;
    int rc = noalloc_job_from_ctx(ctx, env_index, ifreq, &J, &why);
    if(rc != BHCB_OK) return put_msg(msg, msg_len, rc, why ? why : "invalid request");
    const size_t nelem = (size_t)J.nsz * J.nrzp * J.nrr;
    if(bytes < nelem * sizeof(float2)) return put_msg(msg, msg_len, BHCB_ERR_ARG, "output buffer too small");
    // graph scratch, stream and capture on the context's GPU
    DeviceGuard guard(J.device);
    if(!guard.ok) return put_msg(msg, msg_len, BHCB_ERR_CUDA, "cannot make the context's device current");
    auto *g = new bhcb_graph();
    g->device = J.device;
    auto fail = [&](int code, const char *text) {
        cudaGetLastError();
        bhcb_graph_destroy(g);
        return put_msg(msg, msg_len, code, text);
    };
    if(cudaMalloc((void **)&g->scratch, kHeaderBytes + nelem * sizeof(float2)) != cudaSuccess)
        return fail(BHCB_ERR_MEMORY, "graph scratch allocation failed");
    if(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(BHCB_ERR_CUDA, "stream creation failed");
    NoAllocHeader h;
    memset(&h, 0, sizeof h);
    h.ctr.overflow_job = 0xffffffffu;
    h.group = J.group;
    h.group.job_base = 0;
    h.group.nfreq = 1;
    h.group.freq_base = 0;
    h.group.field_base = 0;
    h.group.field_stride_f = (int)nelem;
    h.group.acc_base = 0;
    h.group.acc_stride_f = (int64_t)nelem;
    h.group.acc_nz = J.nrzp;
    J.stream = g->stream;
    long long grid = (J.group.njobs + 31) / 32;
    if(grid > (long long)J.sm_count * 16) grid = (long long)J.sm_count * 16;
    if(grid < 1) grid = 1;
    if(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return fail(BHCB_ERR_CUDA, "stream capture could not begin");
    write_header_kernel<<<1, 64, 0, g->stream>>>(h, g->scratch);
    cudaMemsetAsync(g->scratch + kHeaderBytes, 0, nelem * sizeof(float2), g->stream);
    if(J.precision == BHCB_PREC_FP64) launch_fused<double>(J, g->scratch, (int)grid);
    else launch_fused<float>(J, g->scratch, (int)grid);
    NoAllocHeader *dh = reinterpret_cast<NoAllocHeader *>(g->scratch);
    launch_scale(reinterpret_cast<const float2 *>(g->scratch + kHeaderBytes), (float2 *)field_dev, &dh->group, 1,
                 J.sm_count * 2, g->stream);
    if(cudaStreamEndCapture(g->stream, &g->graph) != cudaSuccess || !g->graph)
        return fail(BHCB_ERR_CUDA, "stream capture failed");
    if(cudaGraphInstantiate(&g->exec, g->graph, 0) != cudaSuccess)
        return fail(BHCB_ERR_CUDA, "graph instantiation failed");
    *out = g;
    return BHCB_OK;
}

extern "C" int bhcb_graph_launch(bhcb_graph *g, void *stream)
{
    if(!g) return BHCB_ERR_ARG;
    cudaStream_t s = stream ? (cudaStream_t)stream : g->stream;
    return cudaGraphLaunch(g->exec, s) == cudaSuccess ? BHCB_OK : BHCB_ERR_CUDA;
}

extern "C" int bhcb_graph_status(bhcb_graph *g, void *stream, uint32_t *err_bits, uint64_t *evals)
{
    if(!g) return BHCB_ERR_ARG;
    cudaStream_t s = stream ? (cudaStream_t)stream : g->stream;
    RunCounters back;
    const NoAllocHeader *dh = reinterpret_cast<const NoAllocHeader *>(g->scratch);
    if(cudaMemcpyAsync(&back, &dh->ctr, sizeof back, cudaMemcpyDeviceToHost, s) != cudaSuccess
       || cudaStreamSynchronize(s) != cudaSuccess)
        return BHCB_ERR_CUDA;
    if(err_bits) *err_bits = back.err_bits;
    if(evals) *evals = back.nevals;
    return back.err_bits ? BHCB_ERR_RUN : BHCB_OK;
}
