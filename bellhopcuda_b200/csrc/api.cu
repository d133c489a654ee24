// Runtime behind the bhcb C ABI: context, environment batch, device arena,
// kernel sequencing and output access. See include/bhcb.h for the contract.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/bhcb.h"
#include "bhcb_internal.h"
#include "host/env2d.h"
#include "host/rt.h"
#include "host/run3d.h"
#include "noalloc.h"
#include "tabstage.cuh"

namespace bhcb {
template<typename R> cudaError_t launch_trace(const GroupDev *, int, long long, void *,
                                              unsigned long long, RunCounters *,
                                              unsigned long long *, unsigned int *, int, int, cudaStream_t,
                                              unsigned int, int);
cudaError_t launch_influence_mixed(const void *, unsigned long long, const GroupDev *, int, const double *,
                                   float2 *, RunCounters *, bool, bool, int, cudaStream_t, unsigned int *,
                                   unsigned long long *);
template<typename R> cudaError_t launch_influence(const void *, unsigned long long,
                                                  const GroupDev *, int, const double *, float2 *,
                                                  RunCounters *, bool, bool, int, cudaStream_t);
cudaError_t launch_scale(const float2 *, float2 *, const GroupDev *, int, int, cudaStream_t);
cudaError_t launch_set_counter(unsigned long long *, unsigned long long, cudaStream_t);
size_t seg_record_bytes(bool fp64);
template<typename R> cudaError_t launch_arr_gather(const void *, unsigned long long, const GroupDev *, int,
                                                   const double *, bool, bool, ArrCand *, uint64_t *, uint32_t *,
                                                   unsigned long long, unsigned long long *, RunCounters *,
                                                   ArrKeyBits, int, cudaStream_t);
cudaError_t launch_arr_gather_x(const XSeg *, unsigned long long, const GroupDev *, int, const double *, int, bool,
                                ArrCand *, uint64_t *, uint32_t *, unsigned long long, unsigned long long *,
                                RunCounters *, ArrKeyBits, int, int, cudaStream_t);
size_t radix_sort_hist_entries(unsigned long long n);
cudaError_t radix_sort_pairs(uint64_t *, uint32_t *, uint64_t *, uint32_t *, unsigned long long, int, uint32_t *,
                             int *, cudaStream_t);
cudaError_t launch_arr_replay(const uint64_t *, const uint32_t *, const ArrCand *, unsigned long long,
                              const GroupDev *, int, const double *, long long, int, int, int, int32_t *,
                              ArrivalRec *, int, cudaStream_t, bool);
cudaError_t launch_rays(const GroupDev *, int, const long long *, const int *, int, const long long *, double2 *, int *,
                        int *, RunCounters *, bool, int, cudaStream_t);
cudaError_t launch_eigen_emit(const uint32_t *, const ArrCand *, unsigned long long, EigenHitRec *, int32_t *, int,
                              const uint64_t *, int, cudaStream_t);
cudaError_t launch_trace_x(const GroupDev *, int, long long, XSeg *, unsigned long long, RunCounters *,
                           unsigned long long *, int, int, int, cudaStream_t);
cudaError_t launch_influence_x(const XSeg *, unsigned long long, const GroupDev *, int, const double *, float2 *,
                               RunCounters *, int, int, int, cudaStream_t);
cudaError_t launch_scale_x(const float2 *, float2 *, const GroupDev *, int, const double *, RunCounters *, int,
                           cudaStream_t);

// influence type of Beam->Type[0] (src/runtype.hpp:150-186)
int infl_kind_of(char bt)
{
    switch(bt) {
    case 'g': case 'b': return INFL_GEO_RAYCEN;
    case 'R': return INFL_CERV_RAYCEN;
    case 'C': return INFL_CERV_CART;
    case 'S': return INFL_SGB;
    default: return INFL_GEO_CART;
    }
}
} // namespace bhcb

using namespace bhcb;

namespace {

struct EnvSlot {
    std::string root;
    EnvInput in;
    std::vector<double> freqs;   // evaluation frequencies (default: file frequency)
    // filled by prepare
    std::vector<EnvTables> tables;    // per frequency
    std::vector<int> field_of_freq;   // global field index per frequency
};

struct Field {
    int env, ifreq;
    int64_t base;        // complex-element offset in out (and receiver-cell offset of arrivals)
    int nsz, nrzp, nrr;
};

// Ray trajectories of one field: every ray of a RunType 'R' run, or the rays
// of its eigen hits re-traced up to the hit; points (r, z) in m, host copies
struct RaySet {
    bool valid = false;
    std::vector<long long> jobs;
    std::vector<int> limits, npts, bnc;   // bnc: top, bottom bounces of the last point
    std::vector<long long> off;
    std::vector<double> alpha_deg;        // take-off angle (SrcDeclAngle)
    std::vector<double> rz;               // 2 doubles per point
};

enum { MODE_TL = 0, MODE_ARR = 1, MODE_EIGEN = 2, MODE_RAY = 3 };
constexpr unsigned long long MAXN_STEPS_HOST = 100000;   // steps per ray (include/bhc/structs.hpp:66)

int run_mode_of(char r0)
{
    if(r0 == 'A' || r0 == 'a' || r0 == 'V' || r0 == 'v') return MODE_ARR;   // 'V' / 'v': also eigen hits
    if(r0 == 'E') return MODE_EIGEN;
    if(r0 == 'C' || r0 == 'S' || r0 == 'I') return MODE_TL;
    if(r0 == 'R') return MODE_RAY;
    throw std::runtime_error(std::string("RunType '") + r0 + "' is not supported by this entry point "
                             "(TL 'C'/'S'/'I', arrivals 'A'/'a', arrivals and eigen hits 'V'/'v', eigen hits 'E', "
                             "rays 'R')");
}

int bits_for(unsigned long long n)   // bits to hold values 0..n-1 (at least 1)
{
    int b = 1;
    while(b < 63 && (1ull << b) < n) ++b;
    return b;
}

} // namespace

struct bhcb_ctx {
    int device = 0;
    int precision = BHCB_PREC_MIXED;
    bool share = true;
    uint64_t max_memory = 16ull << 30;
    void (*output_cb)(const char *) = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;   // influence launches beside the trace
    bool overlap = false;             // mixed TL runs: influence overlaps the trace (BHCB_FLAG_OVERLAP_INFLUENCE)
    // pipelined TL steps (BHCB_FLAG_PIPELINE): slot k % 2 of launch k; slot 0
    // uses segs / counters / acc, slot 1 the pipe_* buffers
    bool pipeline = false;
    cudaStream_t pstream[3] = {nullptr, nullptr, nullptr};   // trace streams of slots 0 / 1, influence stream
    DevBuf pipe_segs, pipe_counters, pipe_acc;
    // per slot: 0 trace start, 1 trace end, 2 influence start, 3 influence end, 4 scale end
    cudaEvent_t pev[2][5] = {};
    cudaEvent_t pev_ctx = nullptr;    // the context stream's position at the first launch
    cudaEvent_t pev_pair = nullptr;   // scale end of the last launch of the previous pair
    long long pipe_k = 0;             // launches since the last prepare
    bool pipe_inflight = false;       // launches not yet waited for by bhcb_sync
    int pipe_used = 0;                // slots (bit mask) launched since the last bhcb_sync
    int pipe_last = 0;                // slot of the last launch
    // the serial TL step captured once into a CUDA graph and replayed
    bool use_graphs = true;
    int graph_state = 0;              // 0: next launch direct, 1: next launch captures, 2: replay
    cudaGraph_t lgraph = nullptr;
    cudaGraphExec_t lexec = nullptr;
    bool capturing = false;           // the step is being captured: events are recorded as external nodes
    // ev: 0 start, 1 trace end, 2 influence end, 3 scale end, 4 first influence launch
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    int sm_count = 148;
    // launch shapes (bhcb_autotune picks them by timing the prepared workload)
    int trace_block = 32;           // threads per trace CTA (one ray each)
    int influence_ctas_per_sm = 8;  // persistent influence CTAs per SM
    int trace_lanes = 32;           // rays per trace warp

    std::vector<EnvSlot> envs;
    bool prepared = false;

    // prepared state
    std::vector<GroupDev> groups_h;
    std::vector<Field> fields;
    std::vector<double> freqs_h;
    int64_t total_field = 0;
    int64_t total_acc = 0;       // accumulator elements (padded rows)
    long long njobs = 0;
    unsigned long long seg_cap = 0;
    bool any_gauss = false, any_coherent = false, mixed_types = false;
    bool gauss = false, coherent = true;
    int xkind = INFL_GEO_CART;       // InflKind of the batch
    unsigned int stage_cap = STAGE_DEFAULT_BYTES;   // staging budget per trace CTA (bhcb_tuning.stage_kb)
    std::vector<EnvDev> envdev_h;    // the prepared environments (counts; plans the staging)

    DevBuf arena, groups_d, freqs_d, acc, out, segs, counters;
    DevBuf blk_state, scan;          // published segment blocks; queue of an overlapped launch
    bool last_overlapped = false;

    // arrivals / eigen runs (RunType 'A', 'a', 'E')
    int mode = MODE_TL;
    bool also_eigen = false;         // RunType 'V' / 'v': an arrivals run that also records eigen hits
    int32_t opt_max_narr = 0, allow_merging = 1;
    int32_t max_narr = 0;
    ArrKeyBits kb{}, kb_eig{};       // ordering keys of the arrivals (or eigen) pass and of the eigen pass of 'V' runs
    unsigned long long ncand = 0;
    DevBuf cand, keys0, keys1, vals0, vals1, hist, narr_d, arr_d, hits_d, hitfield_d;
    const uint64_t *sorted_keys = nullptr;
    const uint32_t *sorted_vals = nullptr;
    std::vector<EigenHitRec> hits_h;      // eigen hits of the last run, in reference order
    std::vector<int64_t> hit_begin;       // per field: first hit (size nfields + 1)
    std::vector<RaySet> rays;             // per field: trajectories (ray runs, eigen re-traces)
    RunCounters last{};
    bhcb_stats stats{};
    std::string last_error;
    uint32_t err_bits = 0, warn_bits = 0;

    // 3-D environments (a context holds either 2-D or 3-D environments)
    Run3 *r3 = nullptr;
    int r3_status = BHCB_OK;
    bool is3d() const { return r3 && run3_count(r3) > 0; }

    void msg(const std::string &s) const
    {
        if(output_cb) output_cb(s.c_str());
    }
};

namespace {

int fail(bhcb_ctx *c, int code, const std::string &m)
{
    if(c) {
        c->last_error = m;
        c->msg(m);
    }
    return code;
}

template<typename F> int guarded(bhcb_ctx *c, F &&fn)
{
    if(!c) return BHCB_ERR_ARG;
    try {
        c->last_error.clear();
        return fn();
    } catch(const CudaError &e) {
        return fail(c, BHCB_ERR_CUDA, e.what());
    } catch(const StateError &e) {
        return fail(c, BHCB_ERR_STATE, e.what());
    } catch(const MemError &e) {
        return fail(c, BHCB_ERR_MEMORY, e.what());
    } catch(const std::exception &e) {
        return fail(c, BHCB_ERR_INPUT, e.what());
    }
}

// Key layout and arrival storage of an arrivals / eigen run.
void prepare_arrivals(bhcb_ctx *c)
{
    int max_njobs = 1, max_nrr = 1, max_nrzp = 1;
    for(const GroupDev &G : c->groups_h) max_njobs = std::max(max_njobs, G.njobs);
    for(const Field &F : c->fields) {
        max_nrr = std::max(max_nrr, F.nrr);
        max_nrzp = std::max(max_nrzp, F.nrzp);
    }
    const int bis = bits_for(MAXN_STEPS_HOST), bjob = bits_for((unsigned long long)max_njobs);
    auto layout = [&](bool eigen) {
        ArrKeyBits kb{};
        if(!eigen) {
            kb.eigen = 0;
            kb.sh_walk = 0;
            kb.sh_is = 0;
            kb.sh_job = bis;
            kb.sh_cell = bis + bjob;
            kb.total_bits = kb.sh_cell + bits_for((unsigned long long)c->total_field);
        } else {
            kb.eigen = 1;
            // within a step: Cartesian and simple Gaussian beams walk the ranges,
            // then the depths; ray-centred beams the depths, then the ranges
            const bool depth_outer = c->xkind == INFL_GEO_RAYCEN;
            const int lo_bits = bits_for((unsigned long long)(depth_outer ? max_nrr : max_nrzp));
            const int hi_bits = bits_for((unsigned long long)(depth_outer ? max_nrzp : max_nrr));
            kb.sh_walk = lo_bits;
            kb.sh_is = kb.sh_walk + hi_bits;
            kb.sh_job = kb.sh_is + bis;
            kb.sh_cell = kb.sh_job + bjob;
            kb.total_bits = kb.sh_cell + bits_for((unsigned long long)c->fields.size());
        }
        if(kb.total_bits > 64)
            throw MemError("arrival ordering key needs more than 64 bits; split the run");
        return kb;
    };
    const ArrKeyBits kb = layout(c->mode != MODE_ARR);
    c->kb_eig = c->also_eigen ? layout(true) : kb;
    c->kb = kb;
    if(c->mode == MODE_ARR) {
        size_t cells = (size_t)c->total_field;
        int32_t mx = c->opt_max_narr;
        if(mx <= 0) {
            // like the reference (src/mode/arr.hpp:80-98): as many arrivals per
            // receiver as a quarter of max_memory holds, at most 1000
            uint64_t m = (c->max_memory / 4) / (cells * sizeof(ArrivalRec) + 1);
            if(c->also_eigen) m /= 2;   // half the room goes to the eigen hits (src/mode/arr.hpp:87)
            mx = (int32_t)std::min<uint64_t>(m, 1000);
        }
        if(mx <= 0) throw MemError("insufficient memory to allocate arrivals");
        c->max_narr = mx;
        c->narr_d.ensure(cells * sizeof(int32_t));
        c->arr_d.ensure(cells * (size_t)mx * sizeof(ArrivalRec));
    }
}

void drop_graph(bhcb_ctx *c);

// Records step event k on stream st; inside a capture as an external event
// node, so that the replayed graph records it like a direct launch does (its
// times stay readable).
cudaError_t record_event(bhcb_ctx *c, int k, cudaStream_t st)
{
    return c->capturing ? cudaEventRecordWithFlags(c->ev[k], st, cudaEventRecordExternal)
                        : cudaEventRecord(c->ev[k], st);
}

void do_prepare(bhcb_ctx *c)
{
    if(c->envs.empty()) throw StateError("no environment: call bhcb_setup or bhcb_add_env first");
    drop_graph(c);
    CK(cudaSetDevice(c->device));
    c->groups_h.clear();
    c->fields.clear();
    c->freqs_h.clear();
    c->total_field = 0;
    c->total_acc = 0;
    c->njobs = 0;
    bool fp64 = c->precision == BHCB_PREC_FP64;
    c->mode = run_mode_of(c->envs[0].in.run_type[0]);
    c->also_eigen = c->envs[0].in.run_type[0] == 'V' || c->envs[0].in.run_type[0] == 'v';
    for(auto &S : c->envs)
        if(run_mode_of(S.in.run_type[0]) != c->mode)
            throw std::runtime_error("a batch must use one run mode (TL, arrivals or eigen hits)");
    // --- preprocess every (env, frequency) and form trace groups
    struct GroupPlan { int env; std::vector<int> ifreqs; };
    std::vector<GroupPlan> plan;
    int nG = 0, nC = 0;
    for(int e = 0; e < (int)c->envs.size(); ++e) {
        EnvSlot &S = c->envs[e];
        S.tables.clear();
        for(double f : S.freqs) S.tables.push_back(preprocess(S.in, f));
        for(const auto &w : S.tables[0].warnings) c->msg("warning: " + w);
        std::vector<bool> done(S.freqs.size(), false);
        for(size_t i = 0; i < S.freqs.size(); ++i) {
            if(done[i]) continue;
            GroupPlan gp{e, {(int)i}};
            done[i] = true;
            if(!fp64 && c->share && c->mode == MODE_TL) {   // arrivals and hits are per frequency
                for(size_t j = i + 1; j < S.freqs.size(); ++j)
                    if(!done[j] && S.tables[i].same_trajectory_tables(S.tables[j])
                       && S.tables[i].alpha == S.tables[j].alpha) {
                        gp.ifreqs.push_back((int)j);
                        done[j] = true;
                    }
            }
            plan.push_back(gp);
        }
        const EnvTables &T0 = S.tables[0];
        char bt = T0.beam_type[0];
        (bt == 'B' ? nG : nC) += 1;
    }
    // one launch handles a single influence flavour; mixed batches are split by the caller
    c->gauss = c->envs[0].tables[0].beam_type[0] == 'B';
    c->xkind = infl_kind_of(c->envs[0].tables[0].beam_type[0]);
    for(auto &S : c->envs)
        if(infl_kind_of(S.tables[0].beam_type[0]) != c->xkind
           || (c->xkind && S.tables[0].beam_type[0] != c->envs[0].tables[0].beam_type[0]))
            throw std::runtime_error("a batch must use one beam type");
    c->coherent = c->envs[0].tables[0].run_type[0] == 'C';
    for(auto &S : c->envs) {
        const EnvTables &T0 = S.tables[0];
        if((T0.beam_type[0] == 'B') != c->gauss || (T0.run_type[0] == 'C') != c->coherent)
            throw std::runtime_error("a batch must use one beam type and one coherence mode");
    }
    // --- build device tables
    Arena A;
    struct EnvOffsets { size_t z, rho, c, cz, n2, n2z, coef, qr, qc, qcz, trc, brc, btop, bbot, rr, rz, sz, alpha, acs, sbp; };
    std::vector<EnvOffsets> offs;
    std::vector<EnvDev> envdev;
    for(const GroupPlan &gp : plan) {
        const EnvSlot &S = c->envs[gp.env];
        const EnvTables &T = S.tables[gp.ifreqs[0]];
        EnvOffsets o;
        o.z = A.put(T.z); o.rho = A.put(T.rho); o.c = A.put(T.c); o.cz = A.put(T.cz);
        o.n2 = A.put(T.n2); o.n2z = A.put(T.n2z); o.coef = A.put(T.coef);
        o.qr = A.put(T.qr); o.qc = A.put(T.qc); o.qcz = A.put(T.qcz);
        o.trc = A.put(T.trc); o.brc = A.put(T.brc);
        o.btop = A.put(T.btop); o.bbot = A.put(T.bbot);
        // depths padded to an even count: the mixed influence kernel reads them in pairs
        std::vector<float> rz_even = T.rz;
        if(rz_even.size() & 1) rz_even.push_back(rz_even.back());
        o.rr = A.put(T.rr); o.rz = A.put(rz_even); o.sz = A.put(T.sz); o.alpha = A.put(T.alpha);
        // launch directions from the host's libm, the same doubles as the
        // reference's RayInit (src/trace.hpp:61) computes on the CPU
        std::vector<double> acs;
        for(double a : T.alpha) { acs.push_back(std::cos(a)); acs.push_back(std::sin(a)); }
        o.acs = A.put(acs);
        o.sbp = A.put(T.sbp);
        offs.push_back(o);
        EnvDev d{};
        d.ssp_type = T.ssp_type;
        d.nssp = (int)T.z.size();
        d.nqr = (int)T.qr.size();
        d.ntrc = (int)(T.trc.size() / 3);
        d.nbrc = (int)(T.brc.size() / 3);
        d.beam_shift = T.beam_type[3] == 'S';
        d.infl_kind = infl_kind_of(T.beam_type[0]);
        d.beam1 = T.beam_type[1];
        d.nimage = T.nimage;
        d.ibeam_window = T.ibeam_window;
        d.component = T.component;
        d.eps_mult = T.eps_mult;
        d.rloop = T.rloop;
        d.top_depth = T.top_depth;
        d.bot_depth = T.bot_depth;
        d.top = T.top;
        d.bot = T.bot;
        d.ntop = (int)T.btop.size();
        d.nbot = (int)T.bbot.size();
        d.top_curv = T.top_curv; d.bot_curv = T.bot_curv;
        d.top_long = T.top_long; d.bot_long = T.bot_long;
        d.nrr = (int)T.rr.size();
        d.nrz = (int)T.rz.size();
        d.nrz_per_range = T.nrz_per_range;
        d.nsz = (int)T.sz.size();
        d.nalpha = (int)T.alpha.size();
        d.isingle = T.isingle;
        d.dalpha = T.dalpha;
        d.delta_r = T.delta_r;
        d.deltas = T.deltas;
        d.box_x = T.box_x;
        d.box_y = T.box_y;
        d.freq0 = T.freq0;
        d.run0 = T.run_type[0];
        d.beam0 = T.beam_type[0];
        d.beam2 = T.beam_type[2];
        d.gaussian = T.beam_type[0] == 'B' || T.beam_type[0] == 'b';   // IsGaussianGeomInfl
        d.coherent = T.run_type[0] == 'C';
        d.line_source = T.run_type[3] == 'X';
        d.irregular = T.run_type[4] == 'I';
        d.q_zero_init = T.run_type[1] == 'G';
        d.nsbp = (int)(T.sbp.size() / 2);
        d.arrivals = c->mode == MODE_ARR;
        envdev.push_back(d);
    }
    c->envdev_h = envdev;
    size_t env_off = A.put(envdev);
    c->arena.ensure(A.bytes.size());
    void *ab = c->arena.p;
    // patch device pointers
    for(size_t g = 0; g < plan.size(); ++g) {
        EnvDev &d = *reinterpret_cast<EnvDev *>(A.bytes.data() + env_off + g * sizeof(EnvDev));
        const EnvOffsets &o = offs[g];
        d.z = dptr<double>(ab, o.z); d.rho = dptr<double>(ab, o.rho);
        d.c = dptr<double>(ab, o.c); d.cz = dptr<double>(ab, o.cz);
        d.n2 = dptr<double>(ab, o.n2); d.n2z = dptr<double>(ab, o.n2z);
        d.coef = dptr<double>(ab, o.coef);
        d.qr = dptr<double>(ab, o.qr); d.qc = dptr<double>(ab, o.qc); d.qcz = dptr<double>(ab, o.qcz);
        d.trc = dptr<double>(ab, o.trc); d.brc = dptr<double>(ab, o.brc);
        d.btop = dptr<BdryPtDev>(ab, o.btop); d.bbot = dptr<BdryPtDev>(ab, o.bbot);
        d.rr = dptr<double>(ab, o.rr); d.rz = dptr<float>(ab, o.rz); d.sz = dptr<float>(ab, o.sz);
        d.alpha = dptr<double>(ab, o.alpha); d.acs = dptr<double>(ab, o.acs); d.sbp = dptr<double>(ab, o.sbp);
    }
    CK(cudaMemcpyAsync(ab, A.bytes.data(), A.bytes.size(), cudaMemcpyHostToDevice, c->stream));
    c->stats.h2d_bytes = A.bytes.size();
    // --- groups, fields, frequencies
    for(auto &S : c->envs) S.field_of_freq.assign(S.freqs.size(), -1);
    for(size_t g = 0; g < plan.size(); ++g) {
        const GroupPlan &gp = plan[g];
        EnvSlot &S = c->envs[gp.env];
        const EnvTables &T = S.tables[gp.ifreqs[0]];
        GroupDev G{};
        G.env = dptr<EnvDev>(ab, env_off + g * sizeof(EnvDev));
        int nal = T.isingle > 0 ? 1 : (int)T.alpha.size();
        G.job_base = c->njobs;
        G.njobs = (int)(nal * T.sz.size());
        G.nfreq = (int)gp.ifreqs.size();
        G.freq_base = (int)c->freqs_h.size();
        G.field_stride_f = (int)(T.sz.size() * T.nrz_per_range * T.rr.size());
        G.field_base = c->total_field;
        G.acc_nz = T.run_type[4] == 'I' ? T.nrz_per_range : (T.nrz_per_range + 1) & ~1;
        G.acc_stride_f = (int64_t)T.sz.size() * T.rr.size() * G.acc_nz;
        c->total_acc = (c->total_acc + 1) & ~int64_t(1);
        G.acc_base = c->total_acc;
        c->total_acc += (int64_t)G.nfreq * G.acc_stride_f;
        G.field_index = (int32_t)c->fields.size();
        for(size_t k = 0; k < gp.ifreqs.size(); ++k) {
            int fi = gp.ifreqs[k];
            c->freqs_h.push_back(S.freqs[fi]);
            Field F{gp.env, fi, c->total_field + (int64_t)k * G.field_stride_f, (int)T.sz.size(),
                    T.nrz_per_range, (int)T.rr.size()};
            S.field_of_freq[fi] = (int)c->fields.size();
            c->fields.push_back(F);
        }
        c->total_field += (int64_t)G.nfreq * G.field_stride_f;
        c->njobs += G.njobs;
        c->groups_h.push_back(G);
    }
    c->groups_d.ensure(c->groups_h.size() * sizeof(GroupDev));
    CK(cudaMemcpyAsync(c->groups_d.p, c->groups_h.data(), c->groups_h.size() * sizeof(GroupDev),
                       cudaMemcpyHostToDevice, c->stream));
    c->stats.h2d_bytes += c->groups_h.size() * sizeof(GroupDev) + c->freqs_h.size() * sizeof(double);
    c->freqs_d.ensure(c->freqs_h.size() * sizeof(double));
    CK(cudaMemcpyAsync(c->freqs_d.p, c->freqs_h.data(), c->freqs_h.size() * sizeof(double),
                       cudaMemcpyHostToDevice, c->stream));
    size_t fbytes = (size_t)c->total_field * sizeof(float2);
    size_t abytes = (size_t)c->total_acc * sizeof(float2);
    c->acc.ensure(abytes);
    c->out.ensure(fbytes);
    c->counters.ensure(sizeof(RunCounters) + 64);
    c->rays.assign(c->fields.size(), RaySet{});
    if(c->mode == MODE_RAY) {   // trajectories only: no segment records
        c->prepared = true;
        return;
    }
    // segment buffer: grows on overflow
    size_t rec = c->xkind ? sizeof(XSeg) : seg_record_bytes(fp64);
    size_t budget = c->max_memory > 2 * fbytes + abytes ? c->max_memory - 2 * fbytes - abytes : 0;
    unsigned long long want = std::max<unsigned long long>(c->seg_cap, (unsigned long long)c->njobs * 1024ull);
    unsigned long long maxcap = budget / rec;
    if(maxcap < 1024) throw MemError("max_memory too small for the segment buffer");
    c->seg_cap = std::min(want, maxcap);
    c->segs.ensure(c->seg_cap * rec);
    if(c->mode != MODE_TL) prepare_arrivals(c);
    c->prepared = true;
}

// Enqueue trace (+ influence and scale for TL runs) of trace groups [g0, g1):
// their jobs are [job_base(g0), job_base(g1)), so the job counter starts at
// job_base(g0). clear: zero the accumulator of those groups first.
void do_launch_range(bhcb_ctx *c, int g0, int g1, bool clear, bool host_driven)
{
    if(!c->prepared) throw StateError("bhcb_launch before bhcb_prepare");
    bool fp64 = c->precision == BHCB_PREC_FP64;
    const int ngall = (int)c->groups_h.size();
    const long long job0 = c->groups_h[g0].job_base;
    const long long job1 = g1 < ngall ? (long long)c->groups_h[g1].job_base : c->njobs;
    // counters cleared, overflow job set to "none", job counter to the first
    // job: memsets and a one-thread kernel, so that a captured step refers to
    // no host memory
    CK(cudaMemsetAsync(c->counters.p, 0, sizeof(RunCounters) + 64, c->stream));
    RunCounters *ctr = (RunCounters *)c->counters.p;
    CK(cudaMemsetAsync(&ctr->overflow_job, 0xff, sizeof(ctr->overflow_job), c->stream));
    unsigned long long *jobc = (unsigned long long *)((uint8_t *)c->counters.p + sizeof(RunCounters));
    if(job0) CK(launch_set_counter(jobc, (unsigned long long)job0, c->stream));
    if(clear) {
        const int64_t a0 = c->groups_h[g0].acc_base;
        const int64_t a1 = g1 < ngall ? c->groups_h[g1].acc_base : c->total_acc;
        CK(cudaMemsetAsync((float2 *)c->acc.p + a0, 0, (size_t)(a1 - a0) * sizeof(float2), c->stream));
    }
    CK(record_event(c, 0, c->stream));
    if(c->xkind) {
        // ray-centred / Cerveny / simple Gaussian beams: FP64 trace with the
        // kind's influence prologue, then its influence kernel and scaling
        const GroupDev *Gx = (const GroupDev *)c->groups_d.p + g0;
        const int ngx = g1 - g0;
        long long xgrid = std::min<long long>((job1 - job0 + 63) / 64, (long long)c->sm_count * 16);
        CK(launch_trace_x(Gx, ngx, job1, (XSeg *)c->segs.p, c->seg_cap, ctr, jobc, c->xkind, (int)std::max(1LL, xgrid),
                          64, c->stream));
        CK(record_event(c, 1, c->stream));
        if(c->mode != MODE_TL) return;   // arrivals / hits: run_arrivals after the trace
        c->last_overlapped = false;
        int nzmax = 1;   // receiver depths per range, the most of the launched groups
        for(int g = g0; g < g1; ++g) nzmax = std::max(nzmax, c->fields[c->groups_h[g].field_index].nrzp);
        CK(launch_influence_x((const XSeg *)c->segs.p, c->seg_cap, Gx, ngx, (const double *)c->freqs_d.p,
                              (float2 *)c->acc.p, ctr, c->xkind, nzmax, c->sm_count * 16, c->stream));
        CK(record_event(c, 2, c->stream));
        CK(launch_scale_x((const float2 *)c->acc.p, (float2 *)c->out.p, Gx, ngx, (const double *)c->freqs_d.p, ctr,
                          c->sm_count * 2, c->stream));
        CK(record_event(c, 3, c->stream));
        return;
    }
    int tblock = c->trace_block;
    unsigned int stage_bytes = 0;   // tables of the launched groups that fit the staging budget
    for(int g = g0; g < g1; ++g) {
        size_t off[ST_COUNT];
        stage_bytes = std::max<unsigned int>(stage_bytes, (unsigned int)stage_plan(c->envdev_h[g], c->stage_cap, off));
    }
    // rays per CTA: trace_lanes of each warp's 32 lanes take rays
    const long long rays_per_cta = std::max(1, tblock * c->trace_lanes / 32);
    long long tgrid = std::min<long long>((job1 - job0 + rays_per_cta - 1) / rays_per_cta, (long long)c->sm_count * 32);
    if(tgrid < 1) tgrid = 1;
    const GroupDev *G = (const GroupDev *)c->groups_d.p + g0;
    int ng = g1 - g0;
    // mixed TL runs driven by the host: influence kernels on stream2 take the
    // segment blocks the trace publishes while it runs (no kernel waits for
    // another; the host relaunches them until the trace's end event)
    const bool ovl = host_driven && c->overlap && !fp64 && c->mode == MODE_TL;
    c->last_overlapped = ovl;
    unsigned int *blk = nullptr;
    if(ovl) {
        const size_t nblk = (size_t)((c->seg_cap + 31) / 32);   // the influence kernel's chunk count
        c->blk_state.ensure(nblk * sizeof(unsigned int));
        c->scan.ensure(64);
        blk = (unsigned int *)c->blk_state.p;
        CK(cudaMemsetAsync(blk, 0, nblk * sizeof(unsigned int), c->stream));
        CK(record_event(c, 0, c->stream));
    }
    if(fp64)
        CK(launch_trace<double>(G, ng, job1, c->segs.p, c->seg_cap, ctr, jobc, blk, (int)tgrid, tblock,
                                c->stream, stage_bytes, c->trace_lanes));
    else
        CK(launch_trace<float>(G, ng, job1, c->segs.p, c->seg_cap, ctr, jobc, blk, (int)tgrid, tblock,
                               c->stream, stage_bytes, c->trace_lanes));
    CK(record_event(c, 1, c->stream));
    if(c->mode != MODE_TL) return;   // arrivals / hits: run_arrivals after the trace
    if(ovl) {
        const int igrid = c->sm_count * c->influence_ctas_per_sm;
        unsigned long long *scan = (unsigned long long *)c->scan.p;
        const double *fq = (const double *)c->freqs_d.p;
        CK(cudaStreamWaitEvent(c->stream2, c->ev[0], 0));
        CK(record_event(c, 4, c->stream2));
        for(;;) {
            cudaError_t q = cudaEventQuery(c->ev[1]);
            if(q == cudaSuccess) break;
            if(q != cudaErrorNotReady) CK(q);
            CK(cudaMemsetAsync(scan, 0, sizeof(unsigned long long), c->stream2));
            CK(launch_influence_mixed(c->segs.p, c->seg_cap, G, ng, fq, (float2 *)c->acc.p, ctr, c->gauss,
                                      c->coherent, igrid, c->stream2, blk, scan));
            CK(cudaStreamSynchronize(c->stream2));
        }
        // the trace has ended: every allocated block is published; take the rest
        CK(cudaStreamWaitEvent(c->stream2, c->ev[1], 0));
        CK(cudaMemsetAsync(scan, 0, sizeof(unsigned long long), c->stream2));
        CK(launch_influence_mixed(c->segs.p, c->seg_cap, G, ng, fq, (float2 *)c->acc.p, ctr, c->gauss,
                                  c->coherent, igrid, c->stream2, blk, scan));
        CK(record_event(c, 2, c->stream2));
        CK(cudaStreamWaitEvent(c->stream, c->ev[2], 0));
        CK(launch_scale((const float2 *)c->acc.p, (float2 *)c->out.p, G, ng, c->sm_count * 2, c->stream));
        CK(record_event(c, 3, c->stream));
        return;
    }
    // the influence grid covers the buffer capacity; chunks past the stored
    // count are skipped by reading the count on the device
    int igrid = c->sm_count * c->influence_ctas_per_sm;   // persistent warps draining the chunk queue
    if(fp64)
        CK(launch_influence<double>(c->segs.p, c->seg_cap, G, ng, (const double *)c->freqs_d.p,
                                    (float2 *)c->acc.p, ctr, c->gauss, c->coherent, igrid, c->stream));
    else
        CK(launch_influence<float>(c->segs.p, c->seg_cap, G, ng, (const double *)c->freqs_d.p,
                                   (float2 *)c->acc.p, ctr, c->gauss, c->coherent, igrid, c->stream));
    CK(record_event(c, 2, c->stream));
    CK(launch_scale((const float2 *)c->acc.p, (float2 *)c->out.p, G, ng, c->sm_count * 2, c->stream));
    CK(record_event(c, 3, c->stream));
}

void do_launch(bhcb_ctx *c, bool host_driven)
{
    do_launch_range(c, 0, (int)c->groups_h.size(), true, host_driven);
}

void drop_graph(bhcb_ctx *c)
{
    // pipelined launches in flight finish first (their slots are rebuilt)
    for(auto &st : c->pstream)
        if(st) cudaStreamSynchronize(st);
    c->pipe_inflight = false;
    c->pipe_k = 0;
    if(c->lexec) cudaGraphExecDestroy(c->lexec);
    if(c->lgraph) cudaGraphDestroy(c->lgraph);
    c->lexec = nullptr;
    c->lgraph = nullptr;
    c->graph_state = 0;
}

// Pipelined TL step (BHCB_FLAG_PIPELINE), geometric Cartesian beams.
// Launches go in pairs: launches 2j and 2j + 1 trace at the same time (each on
// its own stream, into its own slot: segment records, counters, accumulator),
// then their influence and ScalePressure run one after the other on the
// influence stream, and the next pair's traces wait for the pair's last
// scale. Two latency-bound traces share the SMs well (each issues on a few
// per cent of the cycles), while a trace beside an influence launch is
// starved of issue slots, so traces never overlap influences. The context
// stream waits for each launch's fields.
void launch_pipelined(bhcb_ctx *c)
{
    const bool fp64 = c->precision == BHCB_PREC_FP64;
    const int P = (int)(c->pipe_k & 1);
    const size_t seg_bytes = (size_t)c->seg_cap * seg_record_bytes(fp64);
    const size_t ctr_bytes = sizeof(RunCounters) + 64;
    const size_t acc_bytes = (size_t)std::max<int64_t>(c->total_acc, 1) * sizeof(float2);
    if(P == 1) {
        c->pipe_segs.ensure(seg_bytes);
        c->pipe_counters.ensure(ctr_bytes);
        c->pipe_acc.ensure(acc_bytes);
    }
    void *segs = P ? c->pipe_segs.p : c->segs.p;
    RunCounters *ctr = (RunCounters *)(P ? c->pipe_counters.p : c->counters.p);
    float2 *acc = (float2 *)(P ? c->pipe_acc.p : c->acc.p);
    unsigned long long *jobc = (unsigned long long *)((uint8_t *)ctr + sizeof(RunCounters));
    cudaStream_t A = c->pstream[P], Bs = c->pstream[2];
    cudaEvent_t *ev = c->pev[P];
    if(!c->pipe_inflight) {   // the first launch follows the context stream's work
        CK(cudaEventRecord(c->pev_ctx, c->stream));
        for(auto st : c->pstream) CK(cudaStreamWaitEvent(st, c->pev_ctx, 0));
    }
    // the previous pair's influences are done (and with them the slot's last user)
    if(c->pipe_k >= 2) CK(cudaStreamWaitEvent(A, c->pev_pair, 0));
    CK(cudaEventRecord(ev[0], A));
    CK(cudaMemsetAsync(ctr, 0, ctr_bytes, A));
    CK(cudaMemsetAsync(&ctr->overflow_job, 0xff, sizeof(ctr->overflow_job), A));
    CK(cudaMemsetAsync(acc, 0, acc_bytes, A));
    const GroupDev *G = (const GroupDev *)c->groups_d.p;
    const int ng = (int)c->groups_h.size();
    const int tblock = c->trace_block;
    unsigned int stage_bytes = 0;
    for(int g = 0; g < ng; ++g) {
        size_t off[ST_COUNT];
        stage_bytes = std::max<unsigned int>(stage_bytes, (unsigned int)stage_plan(c->envdev_h[g], c->stage_cap, off));
    }
    const long long rays_per_cta = std::max(1, tblock * c->trace_lanes / 32);
    long long tgrid = std::min<long long>((c->njobs + rays_per_cta - 1) / rays_per_cta, (long long)c->sm_count * 32);
    if(tgrid < 1) tgrid = 1;
    if(fp64)
        CK(launch_trace<double>(G, ng, c->njobs, segs, c->seg_cap, ctr, jobc, nullptr, (int)tgrid, tblock, A,
                                stage_bytes, c->trace_lanes));
    else
        CK(launch_trace<float>(G, ng, c->njobs, segs, c->seg_cap, ctr, jobc, nullptr, (int)tgrid, tblock, A,
                               stage_bytes, c->trace_lanes));
    CK(cudaEventRecord(ev[1], A));
    CK(cudaStreamWaitEvent(Bs, ev[1], 0));
    CK(cudaEventRecord(ev[2], Bs));
    const int igrid = c->sm_count * c->influence_ctas_per_sm;
    if(fp64)
        CK(launch_influence<double>(segs, c->seg_cap, G, ng, (const double *)c->freqs_d.p, acc, ctr, c->gauss,
                                    c->coherent, igrid, Bs));
    else
        CK(launch_influence<float>(segs, c->seg_cap, G, ng, (const double *)c->freqs_d.p, acc, ctr, c->gauss,
                                   c->coherent, igrid, Bs));
    CK(cudaEventRecord(ev[3], Bs));
    CK(launch_scale(acc, (float2 *)c->out.p, G, ng, c->sm_count * 2, Bs));
    CK(cudaEventRecord(ev[4], Bs));
    if(P == 1) CK(cudaEventRecord(c->pev_pair, Bs));   // a pair ends
    CK(cudaStreamWaitEvent(c->stream, ev[4], 0));
    c->pipe_last = P;
    c->pipe_used |= 1 << P;
    ++c->pipe_k;
    c->pipe_inflight = true;
    c->last_overlapped = false;
}

// One step of a prepared batch. Serial TL steps run directly the first time
// (one-time kernel set-up happens outside any capture), are captured into a
// CUDA graph the second time, and replay that graph afterwards; whatever
// changes the prepared state or the launch shape drops the graph.
void launch_step(bhcb_ctx *c)
{
    if(c->pipeline && c->mode == MODE_TL && !c->xkind && !c->overlap) {
        launch_pipelined(c);
        return;
    }
    const bool overlapped = c->overlap && c->precision != BHCB_PREC_FP64 && c->mode == MODE_TL;
    if(!c->use_graphs || overlapped || c->mode != MODE_TL || c->graph_state == 0) {
        do_launch(c, c->overlap);
        if(c->use_graphs && !overlapped && c->mode == MODE_TL) c->graph_state = 1;
        return;
    }
    if(c->graph_state == 1) {
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        c->capturing = true;
        try {
            do_launch(c, false);
        } catch(...) {
            c->capturing = false;
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(c->stream, &g);
            if(g) cudaGraphDestroy(g);
            throw;
        }
        c->capturing = false;
        CK(cudaStreamEndCapture(c->stream, &c->lgraph));
        CK(cudaGraphInstantiate(&c->lexec, c->lgraph, 0));
        c->graph_state = 2;
    }
    c->last_overlapped = false;
    CK(cudaGraphLaunch(c->lexec, c->stream));
}

// elapsed time between two recorded events (0 if the pair has no timing)
float event_ms(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0.f;
    if(cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
        cudaGetLastError();
        ms = 0.f;
    }
    return ms;
}

int do_sync(bhcb_ctx *c)
{
    CK(cudaStreamSynchronize(c->stream));
    const bool piped = c->pipe_inflight;
    if(piped) {   // the last pipelined launch: its slot's counters and events
        for(auto &st : c->pstream) CK(cudaStreamSynchronize(st));
        c->pipe_inflight = false;
    }
    const int used = c->pipe_used;
    c->pipe_used = 0;
    const int P = c->pipe_last;
    CK(cudaMemcpy(&c->last, piped && P ? c->pipe_counters.p : c->counters.p, sizeof(RunCounters),
                  cudaMemcpyDeviceToHost));
    if(piped && (used & (1 << (P ^ 1)))) {   // the other slot's launch: its error and warning bits too
        RunCounters o{};
        CK(cudaMemcpy(&o, P ? c->counters.p : c->pipe_counters.p, sizeof(RunCounters), cudaMemcpyDeviceToHost));
        c->last.err_bits |= o.err_bits;
        c->last.warn_bits |= o.warn_bits;
    }
    float t0 = event_ms(c->ev[0], c->ev[1]), t1 = 0, t2 = 0;
    float span = 0;
    if(piped) {
        t0 = event_ms(c->pev[P][0], c->pev[P][1]);
        t1 = event_ms(c->pev[P][2], c->pev[P][3]);
        t2 = event_ms(c->pev[P][0], c->pev[P][4]);
        span = t1;
    } else if(c->mode == MODE_TL) {
        t1 = event_ms(c->ev[1], c->ev[2]);
        t2 = event_ms(c->ev[0], c->ev[3]);
        span = c->last_overlapped ? event_ms(c->ev[4], c->ev[2]) : t1;
    } else {
        t2 = t0;
    }
    c->stats.influence_span_ms = span;
    c->stats.rays = (uint64_t)c->njobs;
    c->stats.steps = c->last.nsteps;
    c->stats.segments = c->last.nseg;
    c->stats.evals = c->last.nevals;
    c->stats.err_bits = c->last.err_bits;
    c->stats.warn_bits = c->last.warn_bits;
    c->stats.groups = (int)c->groups_h.size();
    c->stats.fields = (int)c->fields.size();
    c->stats.trace_ms = t0;
    c->stats.influence_ms = t1;
    c->stats.total_ms = t2;
    c->err_bits = c->last.err_bits;
    c->warn_bits = c->last.warn_bits;
    return 0;
}

// index of the trace group that produces field fi
int group_of_field(const bhcb_ctx *c, int fi)
{
    for(size_t g = 0; g < c->groups_h.size(); ++g) {
        const GroupDev &G = c->groups_h[g];
        if(fi >= G.field_index && fi < G.field_index + G.nfreq) return (int)g;
    }
    throw std::runtime_error("field has no trace group");
}

// Trajectories of R.jobs (limits as for the ray kernel): a count pass sizes
// the point buffer exactly, a second pass of the same deterministic trace
// writes the points; both passes read the context's prepared tables.
void trace_rays(bhcb_ctx *c, RaySet &R)
{
    const int n = (int)R.jobs.size();
    R.npts.assign(n, 0);
    R.bnc.assign(2 * (size_t)n, 0);
    R.off.assign(n, 0);
    R.rz.clear();
    R.valid = true;
    if(n == 0) return;
    DevBuf jobs_d, lim_d, npts_d, bnc_d, off_d, pts_d;
    jobs_d.ensure(n * sizeof(long long));
    lim_d.ensure(n * sizeof(int));
    npts_d.ensure(n * sizeof(int));
    bnc_d.ensure(2 * (size_t)n * sizeof(int));
    off_d.ensure(n * sizeof(long long));
    auto release = [&]() { for(DevBuf *b : {&jobs_d, &lim_d, &npts_d, &bnc_d, &off_d, &pts_d}) b->release(); };
    try {
        CK(cudaMemcpyAsync(jobs_d.p, R.jobs.data(), n * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(lim_d.p, R.limits.data(), n * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemsetAsync(c->counters.p, 0, sizeof(RunCounters), c->stream));
        RunCounters *ctr = (RunCounters *)c->counters.p;
        const GroupDev *G = (const GroupDev *)c->groups_d.p;
        const int ng = (int)c->groups_h.size();
        CK(launch_rays(G, ng, (const long long *)jobs_d.p, (const int *)lim_d.p, n, nullptr, nullptr,
                       (int *)npts_d.p, (int *)bnc_d.p, ctr, true, c->sm_count, c->stream));
        CK(cudaMemcpyAsync(R.npts.data(), npts_d.p, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(R.bnc.data(), bnc_d.p, 2 * (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        RunCounters rc{};
        CK(cudaMemcpyAsync(&rc, ctr, sizeof rc, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if(rc.err_bits) {
            c->err_bits = rc.err_bits;
            throw std::runtime_error("tracer error while tracing rays");
        }
        long long tot = 0;
        for(int i = 0; i < n; ++i) {
            R.off[i] = tot;
            tot += R.npts[i];
        }
        if((size_t)tot * sizeof(double2) > c->max_memory) throw MemError("ray points exceed max_memory");
        pts_d.ensure(std::max<long long>(tot, 1) * sizeof(double2));
        CK(cudaMemcpyAsync(off_d.p, R.off.data(), n * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
        CK(launch_rays(G, ng, (const long long *)jobs_d.p, (const int *)lim_d.p, n, (const long long *)off_d.p,
                       (double2 *)pts_d.p, (int *)npts_d.p, (int *)bnc_d.p, ctr, false, c->sm_count, c->stream));
        R.rz.resize(2 * (size_t)tot);
        if(tot)
            CK(cudaMemcpyAsync(R.rz.data(), pts_d.p, tot * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        c->warn_bits |= rc.warn_bits;
    } catch(...) {
        release();
        R.valid = false;
        throw;
    }
    release();
}

// job index and take-off angle of (isz, ialpha) of trace group G
long long job_of(const bhcb_ctx *c, int g, int isz, int ialpha, double *alpha_deg)
{
    const GroupDev &G = c->groups_h[g];
    const Field &F = c->fields[G.field_index];
    const EnvTables &T = c->envs[F.env].tables[F.ifreq];
    const int nal = T.isingle > 0 ? 1 : (int)T.alpha.size();
    const int local = isz * nal + (T.isingle > 0 ? 0 : ialpha);
    if(alpha_deg) *alpha_deg = (180.0 / 3.14159265358979323846) * T.alpha[ialpha];
    return G.job_base + local;
}

// RunType 'R': every ray of every field (RunRayMode, src/mode/ray.cpp:163-198)
void run_rays(bhcb_ctx *c)
{
    for(size_t fi = 0; fi < c->fields.size(); ++fi) {
        const int g = group_of_field(c, (int)fi);
        const GroupDev &G = c->groups_h[g];
        const Field &F = c->fields[fi];
        const EnvTables &T = c->envs[F.env].tables[F.ifreq];
        const int nal = T.isingle > 0 ? 1 : (int)T.alpha.size();
        RaySet &R = c->rays[fi];
        R = RaySet{};
        for(int local = 0; local < G.njobs; ++local) {
            const int ialpha = T.isingle > 0 ? T.isingle - 1 : local % nal;
            R.jobs.push_back(G.job_base + local);
            R.limits.push_back(-1);
            R.alpha_deg.push_back((180.0 / 3.14159265358979323846) * T.alpha[ialpha]);
        }
        trace_rays(c, R);
    }
    c->stats = bhcb_stats{};
    c->stats.rays = (uint64_t)c->njobs;
    c->stats.fields = (int32_t)c->fields.size();
    c->stats.groups = (int32_t)c->groups_h.size();
}

// eigenray re-trace of field fi's hits (EigenModePostWorker, src/mode/eigen.cpp:24-45)
RaySet &eigen_rays(bhcb_ctx *c, int fi)
{
    RaySet &R = c->rays[fi];
    if(R.valid) return R;
    if(c->hit_begin.size() != c->fields.size() + 1) throw StateError("no hits: run first");
    const int g = group_of_field(c, fi);
    R = RaySet{};
    for(int64_t k = c->hit_begin[fi]; k < c->hit_begin[fi + 1]; ++k) {
        const EigenHitRec &h = c->hits_h[k];
        double a = 0.0;
        R.jobs.push_back(job_of(c, g, h.isz, h.ialpha, &a));
        R.limits.push_back(h.is);
        R.alpha_deg.push_back(a);
    }
    trace_rays(c, R);
    return R;
}

// .ray file (OpenRAYFile / WriteRay, src/mode/ray.hpp:176-247), 2-D, list-directed text
void write_rays(const bhcb_ctx *c, const Field &F, const RaySet &R, const std::string &path)
{
    const EnvSlot &S = c->envs[F.env];
    const EnvTables &T = S.tables[F.ifreq];
    std::ofstream o(path);
    if(!o.good()) throw std::runtime_error("cannot open " + path);
    char b[128];
    o << "'" << S.in.title << "'\n";
    snprintf(b, sizeof b, "%.17g\n", S.freqs[F.ifreq]);
    o << b;
    o << 1 << " " << 1 << " " << T.sz.size() << "\n";
    o << T.alpha.size() << " " << 1 << "\n";
    snprintf(b, sizeof b, "%.17g\n%.17g\n", S.in.ssp_z.empty() ? 0.0 : S.in.ssp_z[0], S.in.bot_depth);
    o << b;
    o << "'rz'\n";
    for(size_t i = 0; i < R.jobs.size(); ++i) {
        if(R.npts[i] <= 0) continue;
        snprintf(b, sizeof b, "%.17g\n", R.alpha_deg[i]);
        o << b;
        o << R.npts[i] << " " << R.bnc[2 * i] << " " << R.bnc[2 * i + 1] << "\n";
        for(int k = 0; k < R.npts[i]; ++k) {
            snprintf(b, sizeof b, "%.17g %.17g\n", R.rz[2 * (R.off[i] + k)], R.rz[2 * (R.off[i] + k) + 1]);
            o << b;
        }
    }
}

// Candidates of the traced segments under key layout kb: count, gather, and
// order them; returns their number (c->sorted_keys / sorted_vals point at the
// order).
unsigned long long gather_sorted(bhcb_ctx *c, const ArrKeyBits &kb)
{
    const bool fp64 = c->precision == BHCB_PREC_FP64;
    const GroupDev *G = (const GroupDev *)c->groups_d.p;
    const int ng = (int)c->groups_h.size();
    const double *fq = (const double *)c->freqs_d.p;
    RunCounters *ctr = (RunCounters *)c->counters.p;
    unsigned long long *cursor = (unsigned long long *)((uint8_t *)c->counters.p + sizeof(RunCounters));
    const int grid = c->sm_count * 16;
    int nzmax = 1;   // receiver depths per range, the most of the batch (ray-centred / simple Gaussian)
    for(const Field &F : c->fields) nzmax = std::max(nzmax, F.nrzp);
    // 1. count
    CK(cudaMemsetAsync(&ctr->nevals, 0, sizeof(unsigned long long), c->stream));
    if(c->xkind)
        CK(launch_arr_gather_x((const XSeg *)c->segs.p, c->seg_cap, G, ng, fq, c->xkind, true, nullptr, nullptr,
                               nullptr, 0, cursor, ctr, kb, nzmax, grid, c->stream));
    else if(fp64)
        CK(launch_arr_gather<double>(c->segs.p, c->seg_cap, G, ng, fq, c->gauss, true, nullptr, nullptr, nullptr, 0,
                                     cursor, ctr, kb, grid, c->stream));
    else
        CK(launch_arr_gather<float>(c->segs.p, c->seg_cap, G, ng, fq, c->gauss, true, nullptr, nullptr, nullptr, 0,
                                    cursor, ctr, kb, grid, c->stream));
    unsigned long long n = 0;
    CK(cudaMemcpyAsync(&n, &ctr->nevals, sizeof n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if(n >= (1ull << 32)) throw MemError("more than 2^32 arrival candidates; split the run");
    const size_t per = sizeof(ArrCand) + 2 * sizeof(uint64_t) + 2 * sizeof(uint32_t);
    if(n * per > c->max_memory) throw MemError("arrival candidates exceed max_memory; raise bhcb_init.max_memory");
    c->ncand = n;
    size_t nn = std::max<size_t>(n, 1);
    c->cand.ensure(nn * sizeof(ArrCand));
    c->keys0.ensure(nn * sizeof(uint64_t));
    c->keys1.ensure(nn * sizeof(uint64_t));
    c->vals0.ensure(nn * sizeof(uint32_t));
    c->vals1.ensure(nn * sizeof(uint32_t));
    c->hist.ensure(radix_sort_hist_entries(nn) * sizeof(uint32_t));
    // 2. gather
    CK(cudaMemsetAsync(cursor, 0, sizeof(unsigned long long), c->stream));
    if(c->xkind)
        CK(launch_arr_gather_x((const XSeg *)c->segs.p, c->seg_cap, G, ng, fq, c->xkind, false, (ArrCand *)c->cand.p,
                               (uint64_t *)c->keys0.p, (uint32_t *)c->vals0.p, n, cursor, ctr, kb, nzmax, grid,
                               c->stream));
    else if(fp64)
        CK(launch_arr_gather<double>(c->segs.p, c->seg_cap, G, ng, fq, c->gauss, false, (ArrCand *)c->cand.p,
                                     (uint64_t *)c->keys0.p, (uint32_t *)c->vals0.p, n, cursor, ctr, kb, grid,
                                     c->stream));
    else
        CK(launch_arr_gather<float>(c->segs.p, c->seg_cap, G, ng, fq, c->gauss, false, (ArrCand *)c->cand.p,
                                    (uint64_t *)c->keys0.p, (uint32_t *)c->vals0.p, n, cursor, ctr, kb, grid,
                                    c->stream));
    // 3. order
    int in1 = 0;
    CK(radix_sort_pairs((uint64_t *)c->keys0.p, (uint32_t *)c->vals0.p, (uint64_t *)c->keys1.p,
                        (uint32_t *)c->vals1.p, n, kb.total_bits, (uint32_t *)c->hist.p, &in1, c->stream));
    c->sorted_keys = (const uint64_t *)(in1 ? c->keys1.p : c->keys0.p);
    c->sorted_vals = (const uint32_t *)(in1 ? c->vals1.p : c->vals0.p);
    return n;
}

// Eigen hits in sorted order, copied to the host with the field of each.
void emit_eigen_hits(bhcb_ctx *c, unsigned long long n, const ArrKeyBits &kb)
{
    const size_t nn = std::max<size_t>(n, 1);
    c->hits_d.ensure(nn * sizeof(EigenHitRec));
    c->hitfield_d.ensure(nn * sizeof(int32_t));
    CK(launch_eigen_emit(c->sorted_vals, (const ArrCand *)c->cand.p, n, (EigenHitRec *)c->hits_d.p,
                         (int32_t *)c->hitfield_d.p, kb.sh_cell, c->sorted_keys, c->sm_count, c->stream));
    c->hits_h.resize(n);
    std::vector<int32_t> fld(n);
    if(n) {
        CK(cudaMemcpyAsync(c->hits_h.data(), c->hits_d.p, n * sizeof(EigenHitRec), cudaMemcpyDeviceToHost,
                           c->stream));
        CK(cudaMemcpyAsync(fld.data(), c->hitfield_d.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    c->hit_begin.assign(c->fields.size() + 1, 0);
    for(size_t k = 0; k < n; ++k) c->hit_begin[fld[k] + 1]++;
    for(size_t f = 0; f < c->fields.size(); ++f) c->hit_begin[f + 1] += c->hit_begin[f];
}

// Arrivals / eigen hits of the traced segments: count, gather, order, replay
// (AddArr) or emit (RecordEigenHit). 'V' / 'v' runs take both passes over the
// same segments, as the reference records the hit of every contribution it
// hands to AddArr (src/influence.hpp:443-450).
void run_arrivals(bhcb_ctx *c)
{
    const GroupDev *G = (const GroupDev *)c->groups_d.p;
    const int ng = (int)c->groups_h.size();
    const double *fq = (const double *)c->freqs_d.p;
    CK(record_event(c, 1, c->stream));
    unsigned long long n = gather_sorted(c, c->kb);
    unsigned long long nevals = n;
    if(c->mode == MODE_ARR) {
        const size_t cells = (size_t)c->total_field;
        CK(cudaMemsetAsync(c->arr_d.p, 0, cells * (size_t)c->max_narr * sizeof(ArrivalRec), c->stream));
        CK(launch_arr_replay(c->sorted_keys, c->sorted_vals, (const ArrCand *)c->cand.p, n, G, ng, fq,
                             (long long)cells, c->kb.sh_cell, c->max_narr, c->allow_merging, (int32_t *)c->narr_d.p,
                             (ArrivalRec *)c->arr_d.p, c->sm_count, c->stream, false));
        if(c->also_eigen) {
            CK(cudaStreamSynchronize(c->stream));   // the replay reads the candidates the eigen pass rewrites
            n = gather_sorted(c, c->kb_eig);
            emit_eigen_hits(c, n, c->kb_eig);
        }
    } else {
        emit_eigen_hits(c, n, c->kb);
    }
    CK(record_event(c, 2, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    float t1 = 0;
    CK(cudaEventElapsedTime(&t1, c->ev[1], c->ev[2]));
    c->stats.influence_ms = t1;
    c->stats.total_ms = c->stats.trace_ms + t1;
    c->stats.evals = nevals;
}

// TL runs whose segments do not fit in max_memory at once: trace the groups in
// contiguous waves, halving a wave (by jobs) until its segments fit.
int run_range(bhcb_ctx *c, int g0, int g1, bhcb_stats &acc)
{
    do_launch_range(c, g0, g1, true, true);
    do_sync(c);
    if(c->last.err_bits & (1u << ERR_SEG_OVERFLOW)) {
        if(g1 - g0 <= 1)
            throw MemError("one environment's segments exceed max_memory; raise bhcb_init.max_memory");
        const long long j0 = c->groups_h[g0].job_base;
        const long long j1 = g1 < (int)c->groups_h.size() ? (long long)c->groups_h[g1].job_base : c->njobs;
        int mid = g0 + 1;
        while(mid < g1 - 1 && c->groups_h[mid].job_base - j0 < (j1 - j0) / 2) ++mid;
        int r = run_range(c, g0, mid, acc);
        if(r) return r;
        return run_range(c, mid, g1, acc);
    }
    if(c->last.err_bits) {
        char b[96];
        snprintf(b, sizeof b, "tracer error bits 0x%x", c->last.err_bits);
        return fail(c, BHCB_ERR_RUN, b);
    }
    acc.steps += c->stats.steps;
    acc.segments += c->stats.segments;
    acc.evals += c->stats.evals;
    acc.warn_bits |= c->stats.warn_bits;
    acc.trace_ms += c->stats.trace_ms;
    acc.influence_ms += c->stats.influence_ms;
    acc.total_ms += c->stats.total_ms;
    acc.groups += 1;   // waves
    return BHCB_OK;
}

int run_waves(bhcb_ctx *c)
{
    bhcb_stats acc{};
    int r = run_range(c, 0, (int)c->groups_h.size(), acc);
    if(r) return r;
    c->stats.steps = acc.steps;
    c->stats.segments = acc.segments;
    c->stats.evals = acc.evals;
    c->stats.warn_bits = c->warn_bits = acc.warn_bits;
    c->stats.err_bits = c->err_bits = 0;
    c->stats.trace_ms = acc.trace_ms;
    c->stats.influence_ms = acc.influence_ms;
    c->stats.total_ms = acc.total_ms;
    c->stats.groups = (int)c->groups_h.size();
    c->msg("segments exceeded max_memory: traced in " + std::to_string(acc.groups) + " waves");
    return BHCB_OK;
}

int run_checked(bhcb_ctx *c)
{
    for(int attempt = 0; attempt < 8; ++attempt) {
        launch_step(c);
        do_sync(c);
        if(c->last.err_bits & (1u << ERR_SEG_OVERFLOW)) {
            // grow the segment buffer and run again
            size_t rec = c->xkind ? sizeof(XSeg) : seg_record_bytes(c->precision == BHCB_PREC_FP64);
            size_t fbytes = (size_t)c->total_field * sizeof(float2);
            size_t abytes = (size_t)c->total_acc * sizeof(float2);
            size_t budget = c->max_memory > 2 * fbytes + abytes ? c->max_memory - 2 * fbytes - abytes : 0;
            unsigned long long maxcap = budget / rec;
            if(c->seg_cap >= maxcap) {
                if(c->mode == MODE_TL && c->groups_h.size() > 1) return run_waves(c);
                throw MemError("segment buffer exceeds max_memory; raise bhcb_init.max_memory");
            }
            c->seg_cap = std::min(maxcap, std::max(c->seg_cap * 2, (unsigned long long)(c->last.nseg * 1.25)));
            c->segs.ensure(c->seg_cap * rec);
            drop_graph(c);   // the segment buffer moved
            continue;
        }
        if(c->last.err_bits) {
            char b[96];
            snprintf(b, sizeof b, "tracer error bits 0x%x", c->last.err_bits);
            return fail(c, BHCB_ERR_RUN, b);
        }
        if(c->mode != MODE_TL) run_arrivals(c);
        return BHCB_OK;
    }
    return fail(c, BHCB_ERR_MEMORY, "segment buffer overflow persisted");
}

const Field *find_field(bhcb_ctx *c, int env, int ifreq)
{
    if(!c->prepared) throw StateError("no run has been prepared");
    if(env < 0 || env >= (int)c->envs.size()) throw std::invalid_argument("env_index out of range");
    const EnvSlot &S = c->envs[env];
    if(ifreq < 0 || ifreq >= (int)S.field_of_freq.size()) throw std::invalid_argument("ifreq out of range");
    return &c->fields[S.field_of_freq[ifreq]];
}

} // namespace

namespace bhcb {
int noalloc_job_from_ctx(bhcb_ctx *c, int32_t env, int32_t ifreq, NoAllocJob *job, const char **why)
{
    if(!c->prepared) { *why = "context not prepared: call bhcb_prepare (or bhcb_run) first"; return BHCB_ERR_STATE; }
    if(c->mode != MODE_TL) { *why = "the context was prepared for arrivals, eigenrays or rays, not a TL field"; return BHCB_ERR_STATE; }
    if(c->xkind) { *why = "this entry point covers geometric Cartesian beams ('G', 'B')"; return BHCB_ERR_ARG; }
    if(env < 0 || env >= (int)c->envs.size()) { *why = "env_index out of range"; return BHCB_ERR_ARG; }
    const EnvSlot &S = c->envs[env];
    if(ifreq < 0 || ifreq >= (int)S.field_of_freq.size()) { *why = "ifreq out of range"; return BHCB_ERR_ARG; }
    const Field &F = c->fields[S.field_of_freq[ifreq]];
    for(const GroupDev &G : c->groups_h) {
        int64_t span = (int64_t)G.nfreq * G.field_stride_f;
        if(F.base >= G.field_base && F.base < G.field_base + span) {
            int k = (int)((F.base - G.field_base) / G.field_stride_f);
            job->group = G;
            job->freq = c->freqs_h[G.freq_base + k];
            job->precision = c->precision;
            job->gaussian = c->gauss;
            job->coherent = c->coherent;
            job->nsz = F.nsz;
            job->nrzp = F.nrzp;
            job->nrr = F.nrr;
            job->sm_count = c->sm_count;
            job->device = c->device;
            job->stream = c->stream;
            return BHCB_OK;
        }
    }
    *why = "field not found in the prepared groups";
    return BHCB_ERR_STATE;
}
} // namespace bhcb

namespace {
// Fortran sequential unformatted records: [int32 n][n bytes][int32 n]
// WriteOutArrivals (src/mode/arr.cpp:88-239), 2-D: binary for RunType 'a',
// list-directed text for 'A'.
void write_arrivals(bhcb_ctx *c, const Field &F, const EnvSlot &S, const EnvTables &T, double freq,
                    const std::string &path)
{
    size_t cells = (size_t)F.nsz * F.nrzp * F.nrr;
    std::vector<int32_t> narr(cells);
    std::vector<ArrivalRec> arr(cells * (size_t)c->max_narr);
    CK(cudaMemcpyAsync(narr.data(), (int32_t *)c->narr_d.p + F.base, cells * sizeof(int32_t),
                       cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(arr.data(), (ArrivalRec *)c->arr_d.p + (size_t)F.base * c->max_narr,
                       arr.size() * sizeof(ArrivalRec), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const double RadDeg = 180.0 / 3.14159265358979323846;
    const bool ascii = T.run_type[0] == 'A' || T.run_type[0] == 'V';
    std::ofstream o(path, std::ios::binary);
    if(!o.good()) throw std::runtime_error("cannot open " + path);
    int nrz = (int)T.rz.size(), nrr = F.nrr, nsz = F.nsz;
    if(ascii) {
        char b[64];
        o << "'2D'\n";
        snprintf(b, sizeof b, "%.9g\n", freq);
        o << b;
        o << nsz;
        for(float v : T.sz) { snprintf(b, sizeof b, " %.9g", v); o << b; }
        o << "\n" << nrz;
        for(float v : T.rz) { snprintf(b, sizeof b, " %.9g", v); o << b; }
        o << "\n" << nrr;
        for(double v : T.rr) { snprintf(b, sizeof b, " %.17g", v); o << b; }
        o << "\n";
    } else {
        RecWriter w(o);
        w.put_bytes("'2D'", 4); w.end();
        w.put((float)freq); w.end();
        w.put((int32_t)nsz); w.put_bytes(T.sz.data(), T.sz.size() * 4); w.end();
        w.put((int32_t)nrz); w.put_bytes(T.rz.data(), T.rz.size() * 4); w.end();
        w.put((int32_t)nrr); w.put_bytes(T.rr.data(), T.rr.size() * 8); w.end();
    }
    RecWriter w(o);
    for(int isz = 0; isz < nsz; ++isz) {
        // MaxNPerSource (src/mode/arr.cpp:24-74): the largest count of this source
        int32_t maxn = 0;
        size_t cb = (size_t)isz * F.nrzp * nrr;
        for(size_t k = 0; k < (size_t)F.nrzp * nrr; ++k) maxn = std::max(maxn, narr[cb + k]);
        if(ascii) o << maxn << "\n";
        else { w.put(maxn); w.end(); }
        for(int iz = 0; iz < F.nrzp; ++iz)
            for(int ir = 0; ir < nrr; ++ir) {
                size_t base = cb + (size_t)iz * nrr + ir;
                int32_t n = narr[base];
                if(ascii) o << n << "\n";
                else { w.put(n); w.end(); }
                for(int a = 0; a < n; ++a) {
                    const ArrivalRec &A = arr[base * c->max_narr + a];
                    float ph = (float)RadDeg * A.Phase;
                    if(ascii) {
                        char b[256];
                        snprintf(b, sizeof b, "%.9g %.9g %.9g %.9g %.9g %.9g %d %d\n", A.a, ph, A.delay_re,
                                 A.delay_im, A.SrcDeclAngle, A.RcvrDeclAngle, A.NTopBnc, A.NBotBnc);
                        o << b;
                    } else {
                        w.put(A.a);
                        w.put((float)(RadDeg * A.Phase));
                        w.put(A.delay_re);
                        w.put(A.delay_im);
                        w.put(A.SrcDeclAngle);
                        w.put(A.RcvrDeclAngle);
                        w.put((float)A.NTopBnc);
                        w.put((float)A.NBotBnc);
                        w.end();
                    }
                }
            }
    }
    (void)S;
}
} // namespace

namespace {
// one complete 3-D run: tables, trace, influence, scale (blocking)
int run3_checked(bhcb_ctx *c)
{
    bhcb_stats st{};
    uint32_t wb = 0;
    const uint32_t eb = run3_run(c->r3, c->stream, c->sm_count, c->max_memory, c->opt_max_narr, c->allow_merging,
                                 c->precision == BHCB_PREC_MIXED, st, wb);
    c->stats = st;
    c->err_bits = eb;
    c->warn_bits = wb;
    if(eb) {
        char b[96];
        snprintf(b, sizeof b, "tracer error bits 0x%x", eb);
        return fail(c, (eb & (1u << ERR_SEG_OVERFLOW)) ? BHCB_ERR_MEMORY : BHCB_ERR_RUN, b);
    }
    return BHCB_OK;
}
} // namespace

extern "C" {

int bhcb_open(const bhcb_init *init, bhcb_ctx **out)
{
    if(!out) return BHCB_ERR_ARG;
    *out = nullptr;
    auto c = std::make_unique<bhcb_ctx>();
    if(init) {
        c->device = init->gpu_index;
        c->precision = init->precision == BHCB_PREC_FP64 ? BHCB_PREC_FP64 : BHCB_PREC_MIXED;
        if(init->max_memory) c->max_memory = init->max_memory;
        c->share = init->share_trajectory != 0;
        c->overlap = (init->flags & BHCB_FLAG_OVERLAP_INFLUENCE) != 0;
        c->use_graphs = (init->flags & BHCB_FLAG_NO_GRAPH) == 0;
        c->pipeline = (init->flags & BHCB_FLAG_PIPELINE) != 0;
        c->output_cb = init->output_callback;
    }
    int ndev = 0;
    if(cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return BHCB_ERR_CUDA;
    }
    if(c->device < 0 || c->device >= ndev) return BHCB_ERR_ARG;
    if(cudaSetDevice(c->device) != cudaSuccess) return BHCB_ERR_CUDA;
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device);
    if(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return BHCB_ERR_CUDA;
    if(cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking) != cudaSuccess) return BHCB_ERR_CUDA;
    for(auto &e : c->ev)
        if(cudaEventCreate(&e) != cudaSuccess) return BHCB_ERR_CUDA;
    if(c->pipeline) {
        for(auto &st : c->pstream)
            if(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return BHCB_ERR_CUDA;
        for(auto &row : c->pev)
            for(auto &e : row)
                if(cudaEventCreate(&e) != cudaSuccess) return BHCB_ERR_CUDA;
        if(cudaEventCreateWithFlags(&c->pev_ctx, cudaEventDisableTiming) != cudaSuccess) return BHCB_ERR_CUDA;
        if(cudaEventCreateWithFlags(&c->pev_pair, cudaEventDisableTiming) != cudaSuccess) return BHCB_ERR_CUDA;
    }
    *out = c.release();
    return BHCB_OK;
}

void bhcb_close(bhcb_ctx *c)
{
    if(!c) return;
    cudaSetDevice(c->device);
    if(c->stream) cudaStreamSynchronize(c->stream);
    drop_graph(c);
    if(c->stream2) cudaStreamSynchronize(c->stream2);
    for(auto &st : c->pstream)
        if(st) cudaStreamSynchronize(st);
    for(DevBuf *b : {&c->arena, &c->groups_d, &c->freqs_d, &c->acc, &c->out, &c->segs, &c->counters, &c->cand,
                     &c->keys0, &c->keys1, &c->vals0, &c->vals1, &c->hist, &c->narr_d, &c->arr_d, &c->hits_d,
                     &c->hitfield_d, &c->blk_state, &c->scan, &c->pipe_segs, &c->pipe_counters, &c->pipe_acc})
        b->release();
    for(auto &e : c->ev)
        if(e) cudaEventDestroy(e);
    for(auto &row : c->pev)
        for(auto &e : row)
            if(e) cudaEventDestroy(e);
    if(c->pev_ctx) cudaEventDestroy(c->pev_ctx);
    if(c->pev_pair) cudaEventDestroy(c->pev_pair);
    for(auto &st : c->pstream)
        if(st) cudaStreamDestroy(st);
    if(c->stream) cudaStreamDestroy(c->stream);
    if(c->stream2) cudaStreamDestroy(c->stream2);
    run3_free(c->r3);
    delete c;
}

int bhcb_clear(bhcb_ctx *c)
{
    return guarded(c, [&]() -> int {
        c->envs.clear();
        c->prepared = false;
        if(c->r3) run3_clear(c->r3);
        return BHCB_OK;
    });
}

int bhcb_add_env(bhcb_ctx *c, const char *root, int32_t *idx)
{
    return guarded(c, [&]() -> int {
        if(!root) throw std::invalid_argument("file_root is NULL");
        if(c->is3d()) throw StateError("the context holds 3-D environments: bhcb_clear first");
        EnvSlot S;
        S.root = root;
        S.in = read_env_files(root);
        S.freqs = {S.in.freq0};
        preprocess(S.in, S.in.freq0);   // validate now, like bhc::setup's Validate pass
        c->envs.push_back(std::move(S));
        c->prepared = false;
        if(idx) *idx = (int32_t)c->envs.size() - 1;
        return BHCB_OK;
    });
}

int bhcb_add_env_desc(bhcb_ctx *c, const bhcb_env_desc *desc, int32_t *idx)
{
    return guarded(c, [&]() -> int {
        if(!desc) throw std::invalid_argument("environment descriptor is NULL");
        if(c->is3d()) throw StateError("the context holds 3-D environments: bhcb_clear first");
        EnvSlot S;
        S.root = "";
        S.in = env_from_desc(*desc);
        S.freqs = {S.in.freq0};
        preprocess(S.in, S.in.freq0);   // validate now, like bhc::setup's Validate pass
        c->envs.push_back(std::move(S));
        c->prepared = false;
        if(idx) *idx = (int32_t)c->envs.size() - 1;
        return BHCB_OK;
    });
}

int bhcb_read_env_desc(const char *root, bhcb_env_desc **desc, char *msg, size_t n)
{
    if(msg && n) msg[0] = 0;
    if(!root || !desc) return BHCB_ERR_ARG;
    *desc = nullptr;
    try {
        EnvInput in = read_env_files(root);
        preprocess(in, in.freq0);   // the same validation as bhcb_add_env
        *desc = desc_from_env(in);
        return BHCB_OK;
    } catch(const std::exception &e) {
        if(msg && n) snprintf(msg, n, "%s", e.what());
        return BHCB_ERR_INPUT;
    }
}

void bhcb_free_env_desc(bhcb_env_desc *desc)
{
    if(desc) free_desc(desc);
}

int bhcb_ssp_at(bhcb_ctx *c, int32_t env, double r, double z, double *cout)
{
    return guarded(c, [&]() -> int {
        if(!cout) throw std::invalid_argument("output pointer is NULL");
        if(env < 0 || env >= (int)c->envs.size()) throw std::invalid_argument("env_index out of range");
        const EnvSlot &S = c->envs[env];
        *cout = ssp_at(preprocess(S.in, S.in.freq0), r, z);
        return BHCB_OK;
    });
}

int bhcb_setup(bhcb_ctx *c, const char *root)
{
    int r = bhcb_clear(c);
    if(r) return r;
    return bhcb_add_env(c, root, nullptr);
}

int bhcb_set_frequencies(bhcb_ctx *c, int32_t env, int32_t n, const double *f)
{
    return guarded(c, [&]() -> int {
        if(env < 0 || env >= (int)c->envs.size()) throw std::invalid_argument("env_index out of range");
        if(n <= 0 || !f) throw std::invalid_argument("need at least one frequency");
        for(int i = 0; i < n; ++i)
            if(!(f[i] > 0.0)) throw std::invalid_argument("frequencies must be positive");
        c->envs[env].freqs.assign(f, f + n);
        c->prepared = false;
        return BHCB_OK;
    });
}

int bhcb_prepare(bhcb_ctx *c)
{
    return guarded(c, [&]() -> int {
        if(c->is3d()) return BHCB_OK;   // 3-D tables are built by the run itself
        do_prepare(c);
        return BHCB_OK;
    });
}

int bhcb_launch(bhcb_ctx *c)
{
    return guarded(c, [&]() -> int {
        if(c->is3d()) {   // 3-D runs complete inside the launch; bhcb_sync reports the status
            c->r3_status = run3_checked(c);
            return BHCB_OK;
        }
        if(!c->prepared) do_prepare(c);
        if(c->mode == MODE_RAY) {   // ray runs complete inside the launch
            run_rays(c);
            return BHCB_OK;
        }
        if(c->mode == MODE_EIGEN || c->also_eigen) c->rays.assign(c->fields.size(), RaySet{});
        launch_step(c);
        return BHCB_OK;
    });
}

int bhcb_sync(bhcb_ctx *c)
{
    return guarded(c, [&]() -> int {
        if(c->is3d()) return c->r3_status;
        if(c->mode == MODE_RAY) return BHCB_OK;
        do_sync(c);
        if(c->last.err_bits) {
            char b[96];
            snprintf(b, sizeof b, "tracer error bits 0x%x", c->last.err_bits);
            return fail(c, (c->last.err_bits & (1u << ERR_SEG_OVERFLOW)) ? BHCB_ERR_MEMORY : BHCB_ERR_RUN, b);
        }
        if(c->mode != MODE_TL) run_arrivals(c);
        return BHCB_OK;
    });
}

int bhcb_run(bhcb_ctx *c)
{
    return guarded(c, [&]() -> int {
        if(c->is3d()) return c->r3_status = run3_checked(c);
        if(!c->prepared) do_prepare(c);
        if(c->mode == MODE_RAY) {
            run_rays(c);
            return BHCB_OK;
        }
        if(c->mode == MODE_EIGEN || c->also_eigen) c->rays.assign(c->fields.size(), RaySet{});
        return run_checked(c);
    });
}

int bhcb_field_shape(bhcb_ctx *c, int32_t env, int32_t *nfreq, int32_t *nsz, int32_t *nrzp, int32_t *nrr)
{
    return guarded(c, [&]() -> int {
        if(c->is3d()) throw StateError("3-D environment: use bhcb_field_shape3d");
        if(env < 0 || env >= (int)c->envs.size()) throw std::invalid_argument("env_index out of range");
        const EnvSlot &S = c->envs[env];
        EnvTables T = S.tables.empty() ? preprocess(S.in, S.freqs[0]) : S.tables[0];
        if(nfreq) *nfreq = (int32_t)S.freqs.size();
        if(nsz) *nsz = (int32_t)T.sz.size();
        if(nrzp) *nrzp = T.nrz_per_range;
        if(nrr) *nrr = (int32_t)T.rr.size();
        return BHCB_OK;
    });
}

int bhcb_copy_field(bhcb_ctx *c, int32_t env, int32_t ifreq, void *dst, size_t bytes)
{
    return guarded(c, [&]() -> int {
        if(c->is3d()) {
            if(ifreq != 0) throw std::invalid_argument("3-D runs have one frequency (ifreq 0)");
            run3_copy_field(c->r3, env, dst, bytes, c->stream);
            return BHCB_OK;
        }
        if(c->mode != MODE_TL) throw StateError("not a TL run: use bhcb_copy_arrivals / bhcb_eigen_hits");
        const Field *F = find_field(c, env, ifreq);
        size_t need = (size_t)F->nsz * F->nrzp * F->nrr * sizeof(float2);
        if(!dst || bytes < need) throw std::invalid_argument("destination too small");
        CK(cudaMemcpyAsync(dst, (float2 *)c->out.p + F->base, need, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return BHCB_OK;
    });
}

int bhcb_field_device(bhcb_ctx *c, int32_t env, int32_t ifreq, void **dptr_out)
{
    return guarded(c, [&]() -> int {
        if(c->is3d()) {
            if(ifreq != 0) throw std::invalid_argument("3-D runs have one frequency (ifreq 0)");
            if(!dptr_out) throw std::invalid_argument("dptr is NULL");
            *dptr_out = run3_field_device(c->r3, env);
            return BHCB_OK;
        }
        const Field *F = find_field(c, env, ifreq);
        if(!dptr_out) throw std::invalid_argument("dptr is NULL");
        *dptr_out = (float2 *)c->out.p + F->base;
        return BHCB_OK;
    });
}

int bhcb_receivers(bhcb_ctx *c, int32_t env, double *rr, int32_t nrr, float *rz, int32_t nrz)
{
    return guarded(c, [&]() -> int {
        if(env < 0 || env >= (int)c->envs.size()) throw std::invalid_argument("env_index out of range");
        const EnvSlot &S = c->envs[env];
        EnvTables T = S.tables.empty() ? preprocess(S.in, S.freqs[0]) : S.tables[0];
        if(rr) std::memcpy(rr, T.rr.data(), std::min<size_t>(nrr, T.rr.size()) * sizeof(double));
        if(rz) std::memcpy(rz, T.rz.data(), std::min<size_t>(nrz, T.rz.size()) * sizeof(float));
        return BHCB_OK;
    });
}

int bhcb_set_arrival_options(bhcb_ctx *c, int32_t max_narr, int32_t allow_merging)
{
    return guarded(c, [&]() -> int {
        if(max_narr < 0) throw std::invalid_argument("max_narr must be >= 0 (0 = sized from max_memory)");
        c->opt_max_narr = max_narr;
        c->allow_merging = allow_merging != 0;
        c->prepared = false;
        return BHCB_OK;
    });
}

int bhcb_arrivals_shape(bhcb_ctx *c, int32_t env, int32_t ifreq, int32_t *nsz, int32_t *nrzp, int32_t *nrr,
                        int32_t *max_narr)
{
    return guarded(c, [&]() -> int {
        if(c->is3d()) {   // 3-D: nsz carries NSz * NSx * NSy * Ntheta, the leading field dimensions
            if(!run3_is_arrivals(c->r3) || c->r3_status != BHCB_OK) throw StateError("no 3-D arrivals run");
            if(ifreq != 0) throw std::invalid_argument("3-D runs have one frequency (ifreq 0)");
            int32_t d[6];
            run3_shape(c->r3, env, d);
            if(nsz) *nsz = d[0] * d[1] * d[2] * d[3];
            if(nrzp) *nrzp = d[4];
            if(nrr) *nrr = d[5];
            if(max_narr) *max_narr = run3_max_narr(c->r3);
            return BHCB_OK;
        }
        if(c->mode != MODE_ARR || !c->prepared) throw StateError("no prepared arrivals run");
        const Field *F = find_field(c, env, ifreq);
        if(nsz) *nsz = F->nsz;
        if(nrzp) *nrzp = F->nrzp;
        if(nrr) *nrr = F->nrr;
        if(max_narr) *max_narr = c->max_narr;
        return BHCB_OK;
    });
}

int bhcb_copy_arrivals(bhcb_ctx *c, int32_t env, int32_t ifreq, int32_t *narr, size_t narr_bytes,
                       bhcb_arrival *arr, size_t arr_bytes)
{
    static_assert(sizeof(bhcb_arrival) == sizeof(ArrivalRec), "arrival record layout");
    return guarded(c, [&]() -> int {
        if(c->is3d()) {
            if(ifreq != 0) throw std::invalid_argument("3-D runs have one frequency (ifreq 0)");
            run3_copy_arrivals(c->r3, env, narr, narr_bytes, arr, arr_bytes, c->stream);
            return BHCB_OK;
        }
        if(c->mode != MODE_ARR || !c->prepared) throw StateError("no arrivals run");
        const Field *F = find_field(c, env, ifreq);
        size_t cells = (size_t)F->nsz * F->nrzp * F->nrr;
        if(narr) {
            if(narr_bytes < cells * sizeof(int32_t)) throw std::invalid_argument("narr buffer too small");
            CK(cudaMemcpyAsync(narr, (int32_t *)c->narr_d.p + F->base, cells * sizeof(int32_t),
                               cudaMemcpyDeviceToHost, c->stream));
        }
        if(arr) {
            size_t need = cells * (size_t)c->max_narr * sizeof(ArrivalRec);
            if(arr_bytes < need) throw std::invalid_argument("arrival buffer too small");
            CK(cudaMemcpyAsync(arr, (ArrivalRec *)c->arr_d.p + (size_t)F->base * c->max_narr, need,
                               cudaMemcpyDeviceToHost, c->stream));
        }
        CK(cudaStreamSynchronize(c->stream));
        return BHCB_OK;
    });
}

int bhcb_eigen_hits(bhcb_ctx *c, int32_t env, int32_t ifreq, bhcb_eigen_hit *hits, int64_t max_hits,
                    int64_t *nhits)
{
    static_assert(sizeof(bhcb_eigen_hit) == sizeof(EigenHitRec), "eigen hit layout");
    return guarded(c, [&]() -> int {
        if(c->is3d()) {
            if(ifreq != 0) throw std::invalid_argument("3-D runs have one frequency (ifreq 0)");
            if(c->r3_status != BHCB_OK) throw StateError("no completed 3-D run");
            const int64_t n = run3_eigen_hits(c->r3, env, hits, hits ? max_hits : 0);
            if(nhits) *nhits = n;
            return BHCB_OK;
        }
        if((c->mode != MODE_EIGEN && !c->also_eigen) || !c->prepared) throw StateError("no eigen-hit run");
        if(env < 0 || env >= (int)c->envs.size()) throw std::invalid_argument("env_index out of range");
        const EnvSlot &S = c->envs[env];
        if(ifreq < 0 || ifreq >= (int)S.field_of_freq.size()) throw std::invalid_argument("ifreq out of range");
        int fi = S.field_of_freq[ifreq];
        if(c->hit_begin.size() != c->fields.size() + 1) throw StateError("no hits: run first");
        int64_t b = c->hit_begin[fi], e = c->hit_begin[fi + 1];
        if(nhits) *nhits = e - b;
        if(hits && max_hits > 0)
            std::memcpy(hits, c->hits_h.data() + b, (size_t)std::min<int64_t>(max_hits, e - b) * sizeof(EigenHitRec));
        return BHCB_OK;
    });
}

int bhcb_writeout(bhcb_ctx *c, int32_t env, int32_t ifreq, const char *root)
{
    return guarded(c, [&]() -> int {
        if(!root) throw std::invalid_argument("file_root is NULL");
        if(c->is3d()) {
            if(ifreq != 0) throw std::invalid_argument("3-D runs have one frequency (ifreq 0)");
            run3_writeout(c->r3, env, root, c->stream);
            return BHCB_OK;
        }
        if(c->mode == MODE_EIGEN || c->mode == MODE_RAY) {   // .ray: traced rays or re-traced eigenrays
            const Field *F = find_field(c, env, ifreq);
            const int fi = (int)(F - c->fields.data());
            const RaySet &R = c->mode == MODE_EIGEN ? eigen_rays(c, fi) : c->rays[fi];
            if(!R.valid) throw StateError("no rays: run first");
            write_rays(c, *F, R, std::string(root) + ".ray");
            return BHCB_OK;
        }
        if(c->mode == MODE_ARR) {
            const Field *F = find_field(c, env, ifreq);
            const EnvSlot &S = c->envs[env];
            write_arrivals(c, *F, S, S.tables[ifreq], S.freqs[ifreq], std::string(root) + ".arr");
            if(c->also_eigen) {   // and the eigenrays (src/api.cpp:465-486)
                const int fi = (int)(F - c->fields.data());
                write_rays(c, *F, eigen_rays(c, fi), std::string(root) + ".ray");
            }
            return BHCB_OK;
        }
        const Field *F = find_field(c, env, ifreq);
        const EnvSlot &S = c->envs[env];
        const EnvTables &T = S.tables[ifreq];
        std::vector<float2> u((size_t)F->nsz * F->nrzp * F->nrr);
        CK(cudaMemcpyAsync(u.data(), (float2 *)c->out.p + F->base, u.size() * sizeof(float2),
                           cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        // .shd layout: src/mode/tl.cpp:38-101 (header), 195-248 (records)
        int nsz = F->nsz, nrz = (int)T.rz.size(), nrr = F->nrr;
        int32_t lrecl = 84;
        lrecl = std::max<int32_t>(lrecl, 2 * 1 * 8);
        lrecl = std::max<int32_t>(lrecl, 1 * 8);
        lrecl = std::max<int32_t>(lrecl, nsz * 4);
        lrecl = std::max<int32_t>(lrecl, nrz * 4);
        lrecl = std::max<int32_t>(lrecl, nrr * 8);
        int nrec = 10 + nsz * F->nrzp;
        std::vector<uint8_t> buf((size_t)lrecl * nrec, 0);
        auto rec = [&](int r) { return buf.data() + (size_t)r * lrecl; };
        int32_t lw = lrecl / 4;
        std::memcpy(rec(0), &lw, 4);
        std::string title = S.in.title;
        title.resize(80, ' ');
        std::memcpy(rec(0) + 4, title.data(), 80);
        const char *pt = T.run_type[4] == 'I' ? "irregular " : "rectilin  ";
        std::memcpy(rec(1), pt, 10);
        int32_t hdr[7] = {1, 1, 1, 1, nsz, nrz, nrr};
        std::memcpy(rec(2), hdr, sizeof hdr);
        double f0 = S.freqs[ifreq], atten = 0.0;
        std::memcpy(rec(2) + 28, &f0, 8);
        std::memcpy(rec(2) + 36, &atten, 8);
        std::memcpy(rec(3), &f0, 8);
        double zero = 0.0;
        std::memcpy(rec(4), &zero, 8);
        std::memcpy(rec(5), &zero, 8); std::memcpy(rec(5) + 8, &zero, 8);
        std::memcpy(rec(6), &zero, 8); std::memcpy(rec(6) + 8, &zero, 8);
        std::memcpy(rec(7), T.sz.data(), nsz * 4);
        std::memcpy(rec(8), T.rz.data(), nrz * 4);
        std::memcpy(rec(9), T.rr.data(), nrr * 8);
        for(int isz = 0; isz < nsz; ++isz)
            for(int iz = 0; iz < F->nrzp; ++iz)
                std::memcpy(rec(10 + isz * F->nrzp + iz), &u[((size_t)isz * F->nrzp + iz) * nrr],
                            (size_t)nrr * 8);
        std::ofstream o(std::string(root) + ".shd", std::ios::binary);
        if(!o.good()) throw std::runtime_error(std::string("cannot open ") + root + ".shd");
        o.write((const char *)buf.data(), buf.size());
        return BHCB_OK;
    });
}

int bhcb_add_env3d(bhcb_ctx *c, const char *root, int32_t *idx)
{
    return guarded(c, [&]() -> int {
        if(!root) throw std::invalid_argument("file_root is NULL");
        if(!c->envs.empty()) throw StateError("the context holds 2-D environments: bhcb_clear first");
        if(!c->r3) c->r3 = run3_new();
        const int i = run3_add_env(c->r3, root);
        c->r3_status = BHCB_OK;
        if(idx) *idx = i;
        return BHCB_OK;
    });
}

int bhcb_setup3d(bhcb_ctx *c, const char *root)
{
    int r = bhcb_clear(c);
    if(r) return r;
    return bhcb_add_env3d(c, root, nullptr);
}

int bhcb_field_shape3d(bhcb_ctx *c, int32_t env, int32_t *dims)
{
    return guarded(c, [&]() -> int {
        if(!c->is3d()) throw StateError("not a 3-D context: use bhcb_field_shape");
        if(!dims) throw std::invalid_argument("dims is NULL");
        run3_shape(c->r3, env, dims);
        return BHCB_OK;
    });
}

int bhcb_grid3d(bhcb_ctx *c, int32_t env, double *sx, double *sy, float *sz, double *rr, float *rz, double *theta)
{
    return guarded(c, [&]() -> int {
        if(!c->is3d()) throw StateError("not a 3-D context");
        std::vector<double> vsx, vsy, vrr, vth;
        std::vector<float> vsz, vrz;
        run3_grid(c->r3, env, vsx, vsy, vsz, vrr, vrz, vth);
        if(sx) std::memcpy(sx, vsx.data(), vsx.size() * sizeof(double));
        if(sy) std::memcpy(sy, vsy.data(), vsy.size() * sizeof(double));
        if(sz) std::memcpy(sz, vsz.data(), vsz.size() * sizeof(float));
        if(rr) std::memcpy(rr, vrr.data(), vrr.size() * sizeof(double));
        if(rz) std::memcpy(rz, vrz.data(), vrz.size() * sizeof(float));
        if(theta) std::memcpy(theta, vth.data(), vth.size() * sizeof(double));
        return BHCB_OK;
    });
}

int bhcb_rays_shape(bhcb_ctx *c, int32_t env, int32_t ifreq, int64_t *nrays, int64_t *npoints)
{
    return guarded(c, [&]() -> int {
        if(c->is3d()) {
            if(ifreq != 0) throw std::invalid_argument("3-D runs have one frequency (ifreq 0)");
            if(c->r3_status != BHCB_OK) throw StateError("no 3-D run");
            int64_t nr = 0, np = 0;
            run3_rays_shape(c->r3, env, c->stream, nr, np);
            if(nrays) *nrays = nr;
            if(npoints) *npoints = np;
            return BHCB_OK;
        }
        if(c->mode != MODE_RAY && c->mode != MODE_EIGEN && !c->also_eigen)
            throw StateError("rays exist for 2-D ray runs ('R') and eigen runs ('E', 'V', 'v')");
        const Field *F = find_field(c, env, ifreq);
        const int fi = (int)(F - c->fields.data());
        const RaySet &R = c->mode != MODE_RAY ? eigen_rays(c, fi) : c->rays[fi];
        if(!R.valid) throw StateError("no rays: run first");
        if(nrays) *nrays = (int64_t)R.jobs.size();
        if(npoints) *npoints = (int64_t)(R.rz.size() / 2);
        return BHCB_OK;
    });
}

int bhcb_copy_rays(bhcb_ctx *c, int32_t env, int32_t ifreq, int32_t *npts, int32_t *bounces, double *alpha_deg,
                   double *rz, size_t rz_bytes)
{
    return guarded(c, [&]() -> int {
        if(c->is3d()) {
            if(ifreq != 0) throw std::invalid_argument("3-D runs have one frequency (ifreq 0)");
            if(c->r3_status != BHCB_OK) throw StateError("no 3-D run");
            run3_copy_rays(c->r3, env, c->stream, npts, bounces, alpha_deg, rz, rz_bytes);
            return BHCB_OK;
        }
        if(c->mode != MODE_RAY && c->mode != MODE_EIGEN && !c->also_eigen)
            throw StateError("rays exist for 2-D ray runs ('R') and eigen runs ('E', 'V', 'v')");
        const Field *F = find_field(c, env, ifreq);
        const int fi = (int)(F - c->fields.data());
        const RaySet &R = c->mode != MODE_RAY ? eigen_rays(c, fi) : c->rays[fi];
        if(!R.valid) throw StateError("no rays: run first");
        if(rz && rz_bytes < R.rz.size() * sizeof(double)) throw std::invalid_argument("rz buffer too small");
        if(npts) std::memcpy(npts, R.npts.data(), R.npts.size() * sizeof(int32_t));
        if(bounces) std::memcpy(bounces, R.bnc.data(), R.bnc.size() * sizeof(int32_t));
        if(alpha_deg) std::memcpy(alpha_deg, R.alpha_deg.data(), R.alpha_deg.size() * sizeof(double));
        if(rz && !R.rz.empty()) std::memcpy(rz, R.rz.data(), R.rz.size() * sizeof(double));
        return BHCB_OK;
    });
}

int bhcb_autotune(bhcb_ctx *c, int32_t repeats, bhcb_tuning *out)
{
    return guarded(c, [&]() -> int {
        if(c->is3d()) throw StateError("the autotuner covers the 2-D TL runs");
        if(!c->prepared) do_prepare(c);
        if(c->mode != MODE_TL) throw StateError("the autotuner covers TL runs");
        if(c->xkind) throw StateError("the autotuner covers geometric Cartesian beams ('G', 'B')");
        const int reps = std::max(1, std::min<int>(repeats, 16));
        const bool overlap = c->overlap, graphs = c->use_graphs, pipeline = c->pipeline;
        c->overlap = false;   // time the trace and the influence separately
        c->use_graphs = false;   // every shape launched directly
        drop_graph(c);        // (also drains pipelined launches)
        c->pipeline = false;  // one launch at a time on the context stream
        auto timed = [&](double &tr, double &inf) {
            tr = inf = 1e300;
            for(int r = 0; r < reps; ++r) {
                if(run_checked(c) != BHCB_OK) throw std::runtime_error("run failed while tuning");
                tr = std::min(tr, c->stats.trace_ms);
                inf = std::min(inf, c->stats.influence_ms);
            }
        };
        bhcb_tuning t{};
        t.trace_block = c->trace_block;
        t.influence_ctas_per_sm = c->influence_ctas_per_sm;
        double tr = 0, inf = 0;
        timed(tr, inf);   // warm-up and the current shape
        t.trace_ms = tr;
        t.influence_ms = inf;
        for(int tb : {32, 64}) {   // the trace kernel is compiled for at most 64 threads per CTA
            c->trace_block = tb;
            timed(tr, inf);
            if(tr < t.trace_ms) { t.trace_ms = tr; t.trace_block = tb; }
        }
        c->trace_block = t.trace_block;
        t.trace_lanes = c->trace_lanes;
        for(int ln : {16, 32}) {   // rays per trace warp: 16 diverge less, if the warps fit
            c->trace_lanes = ln;
            timed(tr, inf);
            if(tr < t.trace_ms) { t.trace_ms = tr; t.trace_lanes = ln; }
        }
        c->trace_lanes = t.trace_lanes;
        t.stage_kb = (int32_t)(c->stage_cap / 1024);
        for(int kb : {0, 32, 64}) {   // shared-memory table staging
            c->stage_cap = (unsigned int)kb * 1024u;
            timed(tr, inf);
            if(tr < t.trace_ms) { t.trace_ms = tr; t.stage_kb = kb; }
        }
        c->stage_cap = (unsigned int)t.stage_kb * 1024u;
        for(int k : {2, 3, 4, 5, 6, 8, 10, 12}) {
            c->influence_ctas_per_sm = k;
            timed(tr, inf);
            if(inf < t.influence_ms) { t.influence_ms = inf; t.influence_ctas_per_sm = k; }
        }
        c->influence_ctas_per_sm = t.influence_ctas_per_sm;
        c->overlap = overlap;
        c->use_graphs = graphs;
        c->pipeline = pipeline;
        drop_graph(c);
        if(out) *out = t;
        char b[160];
        snprintf(b, sizeof b, "autotune: trace %d threads/CTA, %d rays/warp, %d KB staged (%.3f ms), influence %d CTAs/SM "
                 "(%.3f ms)", t.trace_block, t.trace_lanes, t.stage_kb, t.trace_ms, t.influence_ctas_per_sm,
                 t.influence_ms);
        c->msg(b);
        return BHCB_OK;
    });
}

int bhcb_set_tuning(bhcb_ctx *c, const bhcb_tuning *t)
{
    return guarded(c, [&]() -> int {
        if(!t) throw std::invalid_argument("tuning is NULL");
        if(t->trace_block != 32 && t->trace_block != 64) throw std::invalid_argument("trace_block must be 32 or 64");
        if(t->influence_ctas_per_sm < 1 || t->influence_ctas_per_sm > 64)
            throw std::invalid_argument("influence_ctas_per_sm must be in 1..64");
        if(t->stage_kb < 0 || t->stage_kb > (int32_t)(STAGE_MAX_BYTES / 1024))
            throw std::invalid_argument("stage_kb must be in 0..64");
        if(t->trace_lanes != 0 && t->trace_lanes != 16 && t->trace_lanes != 32)
            throw std::invalid_argument("trace_lanes must be 16 or 32 (0: 32)");
        c->trace_block = t->trace_block;
        c->influence_ctas_per_sm = t->influence_ctas_per_sm;
        c->stage_cap = (unsigned int)t->stage_kb * 1024u;
        c->trace_lanes = t->trace_lanes ? t->trace_lanes : 32;
        drop_graph(c);
        return BHCB_OK;
    });
}

int bhcb_stream(bhcb_ctx *c, void **stream)
{
    if(!c || !stream) return BHCB_ERR_ARG;
    *stream = (void *)c->stream;
    return BHCB_OK;
}

int bhcb_get_stats(bhcb_ctx *c, bhcb_stats *s)
{
    if(!c || !s) return BHCB_ERR_ARG;
    *s = c->stats;
    return BHCB_OK;
}

int bhcb_last_error(bhcb_ctx *c, char *msg, size_t n, uint32_t *eb, uint32_t *wb)
{
    if(!c) return BHCB_ERR_ARG;
    if(msg && n) {
        size_t l = std::min(n - 1, c->last_error.size());
        std::memcpy(msg, c->last_error.data(), l);
        msg[l] = 0;
    }
    if(eb) *eb = c->err_bits;
    if(wb) *wb = c->warn_bits;
    return BHCB_OK;
}

int bhcb_check_env3d(const char *root, int32_t *dims, int64_t *nrays, char *msg, size_t n)
{
    try {
        if(!root) throw std::invalid_argument("file_root is NULL");
        EnvInput in = read_env_files(root, true);
        Env3Tables T = preprocess3d(in, in.freq0);
        if(dims) {
            dims[0] = (int32_t)T.sz.size(); dims[1] = (int32_t)T.sx.size(); dims[2] = (int32_t)T.sy.size();
            dims[3] = (int32_t)T.theta.size(); dims[4] = (int32_t)T.rz.size(); dims[5] = (int32_t)T.rr.size();
        }
        if(nrays) {
            int64_t r = (int64_t)T.sz.size() * T.sx.size() * T.sy.size();
            if(T.isingle_alpha == 0) r *= (int64_t)T.alpha.size();
            if(T.isingle_beta == 0) r *= (int64_t)T.beta.size();
            *nrays = r;
        }
        if(msg && n) msg[0] = 0;
        return BHCB_OK;
    } catch(const std::exception &e) {
        if(msg && n) {
            size_t l = std::min(n - 1, std::strlen(e.what()));
            std::memcpy(msg, e.what(), l);
            msg[l] = 0;
        }
        return BHCB_ERR_INPUT;
    }
}

int bhcb_check_env(const char *root, bhcb_env_info *info, char *msg, size_t n)
{
    try {
        if(!root) throw std::invalid_argument("file_root is NULL");
        EnvInput in = read_env_files(root);
        EnvTables T = preprocess(in, in.freq0);
        if(info) {
            std::memset(info, 0, sizeof(*info));
            info->nsz = (int32_t)T.sz.size();
            info->nrz = (int32_t)T.rz.size();
            info->nrz_per_range = T.nrz_per_range;
            info->nrr = (int32_t)T.rr.size();
            info->nalpha = (int32_t)T.alpha.size();
            info->ssp_type = T.ssp_type;
            info->freq = T.freq0;
            info->deltas = T.deltas;
            std::memcpy(info->run_type, T.run_type, 7);
            std::memcpy(info->beam_type, T.beam_type, 4);
        }
        if(msg && n) msg[0] = 0;
        return BHCB_OK;
    } catch(const std::exception &e) {
        if(msg && n) {
            size_t l = std::min(n - 1, std::strlen(e.what()));
            std::memcpy(msg, e.what(), l);
            msg[l] = 0;
        }
        return BHCB_ERR_INPUT;
    }
}

const char *bhcb_version(void) { return "bhcb 0.1 (sm_100a)"; }

} // extern "C"
