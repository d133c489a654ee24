// 3-D runner behind the bhcb C ABI (BELLHOP3D field modes): environment batch,
// device tables, trace -> influence -> scale sequencing, field output.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "bhcb_internal.h"
#include "host/env2d.h"
#include "host/rt.h"
#include "host/run3d.h"

namespace bhcb {

cudaError_t launch_arr_gather3d_rc(const XSeg3 *, unsigned long long, const GroupDev *, int, bool, ArrCand *,
                                   uint64_t *, uint32_t *, unsigned long long, unsigned long long *, RunCounters *,
                                   ArrKeyBits, int, int, cudaStream_t);
cudaError_t launch_rays_nx(const GroupDev *, int, const long long *, const int *, int, const long long *, double *,
                           int *, int *, RunCounters *, bool, int, cudaStream_t);
cudaError_t launch_rays3d(const GroupDev *, int, const long long *, const int *, int, const long long *, double *,
                          int *, int *, RunCounters *, bool, int, cudaStream_t);
cudaError_t launch_trace3d_rc(const GroupDev *, int, long long, XSeg3 *, unsigned long long, RunCounters *,
                              unsigned long long *, int, cudaStream_t);
cudaError_t launch_influence3d_rc(const XSeg3 *, unsigned long long, const GroupDev *, int, float2 *, RunCounters *,
                                  int, int, cudaStream_t);
cudaError_t launch_trace_nx(const GroupDev *, int, long long, void *, unsigned long long, RunCounters *,
                            unsigned long long *, int, cudaStream_t);
cudaError_t launch_arr_gather_nx(const void *, unsigned long long, const GroupDev *, int, bool, ArrCand *,
                                 uint64_t *, uint32_t *, unsigned long long, unsigned long long *, RunCounters *,
                                 ArrKeyBits, int, cudaStream_t);
cudaError_t launch_influence_nx(const void *, unsigned long long, const GroupDev *, int, float2 *, RunCounters *, int,
                                int, cudaStream_t);
cudaError_t launch_scale_nx(float2 *, const GroupDev *, int, int, cudaStream_t);
size_t nx_record_bytes();
cudaError_t launch_trace3d(const GroupDev *, int, long long, SegRec3 *, unsigned long long, RunCounters *,
                           unsigned long long *, int, cudaStream_t);
cudaError_t launch_influence3d(const SegRec3 *, unsigned long long, const GroupDev *, int, float2 *, RunCounters *,
                               int, cudaStream_t, bool);
cudaError_t launch_sqrt3d(float2 *, long long, int, cudaStream_t);
cudaError_t launch_arr_gather3d(const SegRec3 *, unsigned long long, const GroupDev *, int, bool, ArrCand *,
                                uint64_t *, uint32_t *, unsigned long long, unsigned long long *, RunCounters *,
                                ArrKeyBits, int, cudaStream_t);
size_t radix_sort_hist_entries(unsigned long long n);
cudaError_t radix_sort_pairs(uint64_t *, uint32_t *, uint64_t *, uint32_t *, unsigned long long, int, uint32_t *,
                             int *, cudaStream_t);
cudaError_t launch_eigen_emit3(const uint32_t *, const ArrCand *, unsigned long long, const GroupDev *, int,
                               EigenHitRec *, int32_t *, int, cudaStream_t);
cudaError_t launch_arr_replay(const uint64_t *, const uint32_t *, const ArrCand *, unsigned long long,
                              const GroupDev *, int, const double *, long long, int, int, int, int32_t *,
                              ArrivalRec *, int, cudaStream_t, bool);

namespace {
struct Env3Slot {
    std::string root;
    EnvInput in;
    Env3Tables T;
    int64_t field_base = 0, field_n = 0;
};

// Trajectories of listed rays of one environment (RunType 'R': all of them;
// 'E': the hit rays, each up to its hit step)
struct RaySet3 {
    bool valid = false;
    std::vector<long long> jobs;
    std::vector<int> limits, npts, bnc;   // bnc: top, bottom bounces of the last point
    std::vector<long long> off;
    std::vector<double> alpha_deg;        // take-off declination (SrcDeclAngle)
    std::vector<double> xyz;              // 3 doubles per point
};
} // namespace

struct Run3 {
    std::vector<Env3Slot> envs;
    std::vector<GroupDev> groups_h;
    DevBuf arena, groups_d, segs, counters, field;
    long long njobs = 0;
    unsigned long long seg_cap = 0;
    int64_t total_field = 0;   // receiver cells of the batch
    bool ran = false;
    // arrivals runs (RunType 'A' / 'a') and eigen-hit runs ('E')
    bool arrivals = false, eigen = false;
    bool also_eigen = false;          // 'V' / 'v': an arrivals run that also records the eigen hits
    ArrKeyBits kb_eig{};              // the eigen pass of 'V' / 'v' runs
    std::vector<EigenHitRec> hits_h;   // in the reference's single-threaded order
    std::vector<int32_t> hit_group;    // environment of each hit
    DevBuf hits_d, hitgrp_d;
    int32_t opt_max_narr = 0, max_narr = 0, allow_merging = 1;
    uint64_t max_memory = 16ull << 30;
    ArrKeyBits kb{};
    DevBuf narr_d, arr_d, cand, keys0, keys1, vals0, vals1, hist;
    // ray runs ('R'), and the eigenray re-trace of 'E' runs
    bool rayrun = false;
    std::vector<RaySet3> raysets;     // per environment
    bool raycen = false;              // geometric beams in ray-centred coordinates ('g', 'b')
    bool nx2d = false;                // N x 2-D rays (RunType(6) '2')
    bool mixed = false;               // Cartesian TL contributions in mixed precision (BHCB_PREC_MIXED)
    int sm_count = 148;
};

Run3 *run3_new() { return new Run3(); }

void run3_free(Run3 *r)
{
    if(!r) return;
    for(DevBuf *b : {&r->arena, &r->groups_d, &r->segs, &r->counters, &r->field, &r->narr_d, &r->arr_d, &r->cand,
                     &r->keys0, &r->keys1, &r->vals0, &r->vals1, &r->hist, &r->hits_d, &r->hitgrp_d})
        b->release();
    delete r;
}

void run3_clear(Run3 *r)
{
    r->envs.clear();
    r->ran = false;
}

int run3_count(const Run3 *r) { return (int)r->envs.size(); }

int run3_add_env(Run3 *r, const std::string &root)
{
    Env3Slot S;
    S.root = root;
    S.in = read_env_files(root, true);
    S.T = preprocess3d(S.in, S.in.freq0);
    r->envs.push_back(std::move(S));
    r->ran = false;
    return (int)r->envs.size() - 1;
}

namespace {

int64_t rays_of(const Env3Tables &T)
{
    int64_t n = 1;
    if(T.isingle_alpha == 0) n *= (int64_t)T.alpha.size();
    if(T.isingle_beta == 0) n *= (int64_t)T.beta.size();
    return n * (int64_t)T.sy.size() * (int64_t)T.sx.size() * (int64_t)T.sz.size();
}

int64_t field_elems(const Env3Tables &T)
{
    return (int64_t)T.sz.size() * T.sx.size() * T.sy.size() * T.theta.size() * T.rz.size() * T.rr.size();
}

void prepare3(Run3 *r, cudaStream_t st, uint64_t &h2d)
{
    if(r->envs.empty()) throw StateError("no 3-D environment: call bhcb_setup3d first");
    Arena A;
    struct Offs { size_t z, rho, c, cz, n2, n2z, coef, hx, hy, hz, hc, hcz, btop, bbot, sx, sy, sz, rr, rz, tcs,
                  alpha, beta, acs, bcs, sbp, trc, brc; };
    std::vector<Offs> offs;
    std::vector<Env3Dev> envdev;
    r->groups_h.clear();
    r->njobs = 0;
    r->total_field = 0;
    for(auto &S : r->envs) {
        const Env3Tables &T = S.T;
        Offs o;
        o.z = A.put(T.z); o.rho = A.put(T.rho); o.c = A.put(T.c); o.cz = A.put(T.cz);
        o.n2 = A.put(T.n2); o.n2z = A.put(T.n2z); o.coef = A.put(T.coef);
        o.hx = A.put(T.hx); o.hy = A.put(T.hy); o.hz = A.put(T.hz); o.hc = A.put(T.hc); o.hcz = A.put(T.hcz);
        std::vector<Bdry3PtDev> bt(T.btop.size()), bb(T.bbot.size());
        static_assert(sizeof(Bdry3PtDev) == sizeof(Bdry3Pt), "3-D boundary node layouts differ");
        if(!bt.empty()) std::memcpy(bt.data(), T.btop.data(), bt.size() * sizeof(Bdry3PtDev));
        if(!bb.empty()) std::memcpy(bb.data(), T.bbot.data(), bb.size() * sizeof(Bdry3PtDev));
        o.btop = A.put(bt); o.bbot = A.put(bb);
        o.sx = A.put(T.sx); o.sy = A.put(T.sy); o.sz = A.put(T.sz); o.rr = A.put(T.rr); o.rz = A.put(T.rz);
        // receiver bearing directions (src/module/rcvrbearings.hpp:103-111)
        std::vector<double> tcs;
        for(double th : T.theta) {
            const double a = (M_PI / 180.0) * th;
            tcs.push_back(std::cos(a));
            tcs.push_back(std::sin(a));
        }
        o.tcs = A.put(tcs);
        o.alpha = A.put(T.alpha); o.beta = A.put(T.beta); o.sbp = A.put(T.sbp);
        // launch directions as the host's libm gives them, so that the Nx2D
        // planes (cos beta, sin beta) are the same doubles as the reference's
        std::vector<double> acs, bcs;
        for(double a : T.alpha) { acs.push_back(std::cos(a)); acs.push_back(std::sin(a)); }
        for(double b : T.beta) { bcs.push_back(std::cos(b)); bcs.push_back(std::sin(b)); }
        o.acs = A.put(acs); o.bcs = A.put(bcs);
        o.trc = A.put(T.trc); o.brc = A.put(T.brc);
        offs.push_back(o);

        Env3Dev d{};
        d.nx2d = T.nx2d ? 1 : 0;
        EnvDev &e = d.e1d;
        e.ssp_type = T.ssp_type == SSP_HEXAHEDRAL ? SSP_CLINEAR : T.ssp_type;
        e.nssp = (int)T.z.size();
        e.top = T.top;
        e.bot = T.bot;
        e.freq0 = T.freq0;
        e.deltas = T.deltas;
        e.ntrc = (int)(T.trc.size() / 3);
        e.nbrc = (int)(T.brc.size() / 3);
        // the plane's receiver ranges and beam flags for the 2-D influence of Nx2D rays
        e.nrr = (int)T.rr.size();
        e.gaussian = T.beam_type[0] == 'B';
        e.coherent = T.run_type[0] == 'C';
        e.beam2 = T.beam_type[2];
        e.run0 = T.run_type[0];
        e.arrivals = T.nx2d && (T.run_type[0] == 'A' || T.run_type[0] == 'a' || T.run_type[0] == 'V' ||
                                T.run_type[0] == 'v');   // records carry the receiver angle
        d.hex = T.ssp_type == SSP_HEXAHEDRAL;
        d.hnx = (int)T.hx.size(); d.hny = (int)T.hy.size(); d.hnz = (int)T.hz.size();
        d.top = T.top;
        d.bot = T.bot;
        d.top_nx = T.top_nx; d.top_ny = T.top_ny; d.bot_nx = T.bot_nx; d.bot_ny = T.bot_ny;
        d.top_curv = T.top_curv; d.bot_curv = T.bot_curv;
        d.nsx = (int)T.sx.size(); d.nsy = (int)T.sy.size(); d.nsz = (int)T.sz.size();
        d.nrr = (int)T.rr.size(); d.nrz = (int)T.rz.size(); d.ntheta = (int)T.theta.size();
        d.nalpha = (int)T.alpha.size(); d.nbeta = (int)T.beta.size();
        d.isingle_alpha = T.isingle_alpha; d.isingle_beta = T.isingle_beta;
        d.dalpha = T.dalpha; d.dbeta = T.dbeta; d.deltas = T.deltas;
        d.box_x = T.box_x; d.box_y = T.box_y; d.box_z = T.box_z; d.freq0 = T.freq0;
        d.gaussian = T.beam_type[0] == 'B' || T.beam_type[0] == 'b';   // IsGaussianGeomInfl
        d.coherent = T.run_type[0] == 'C';
        d.run0 = T.run_type[0];
        d.nsbp = (int)(T.sbp.size() / 2);
        envdev.push_back(d);

        GroupDev g{};
        g.env = nullptr;
        g.job_base = r->njobs;
        const int64_t nj = rays_of(T);
        if(nj > (int64_t)0x7fffffff) throw std::runtime_error("too many rays in one 3-D environment");
        g.njobs = (int32_t)nj;
        g.nfreq = 1;
        g.field_base = r->total_field;
        S.field_base = r->total_field;
        S.field_n = field_elems(T);
        g.field_stride_f = (int32_t)std::min<int64_t>(S.field_n, 0x7fffffff);
        r->groups_h.push_back(g);
        r->njobs += nj;
        r->total_field += S.field_n;
    }
    const size_t env_off = A.put(envdev);
    r->arena.ensure(A.bytes.size());
    void *ab = r->arena.p;
    for(size_t i = 0; i < r->envs.size(); ++i) {
        Env3Dev &d = *reinterpret_cast<Env3Dev *>(A.bytes.data() + env_off + i * sizeof(Env3Dev));
        const Offs &o = offs[i];
        EnvDev &e = d.e1d;
        e.z = dptr<double>(ab, o.z); e.rho = dptr<double>(ab, o.rho);
        e.c = dptr<double>(ab, o.c); e.cz = dptr<double>(ab, o.cz);
        e.n2 = dptr<double>(ab, o.n2); e.n2z = dptr<double>(ab, o.n2z); e.coef = dptr<double>(ab, o.coef);
        e.trc = dptr<double>(ab, o.trc); e.brc = dptr<double>(ab, o.brc);
        e.rr = dptr<double>(ab, o.rr);
        d.hx = dptr<double>(ab, o.hx); d.hy = dptr<double>(ab, o.hy); d.hz = dptr<double>(ab, o.hz);
        d.hc = dptr<double>(ab, o.hc); d.hcz = dptr<double>(ab, o.hcz);
        d.btop = dptr<Bdry3PtDev>(ab, o.btop); d.bbot = dptr<Bdry3PtDev>(ab, o.bbot);
        d.sx = dptr<double>(ab, o.sx); d.sy = dptr<double>(ab, o.sy); d.sz = dptr<float>(ab, o.sz);
        d.rr = dptr<double>(ab, o.rr); d.rz = dptr<float>(ab, o.rz); d.tcs = dptr<double>(ab, o.tcs);
        d.alpha = dptr<double>(ab, o.alpha); d.beta = dptr<double>(ab, o.beta); d.sbp = dptr<double>(ab, o.sbp);
        d.acs = dptr<double>(ab, o.acs); d.bcs = dptr<double>(ab, o.bcs);
        r->groups_h[i].env3 = dptr<Env3Dev>(ab, env_off + i * sizeof(Env3Dev));
    }
    CK(cudaMemcpyAsync(ab, A.bytes.data(), A.bytes.size(), cudaMemcpyHostToDevice, st));
    r->groups_d.ensure(r->groups_h.size() * sizeof(GroupDev));
    CK(cudaMemcpyAsync(r->groups_d.p, r->groups_h.data(), r->groups_h.size() * sizeof(GroupDev),
                       cudaMemcpyHostToDevice, st));
    r->counters.ensure(sizeof(RunCounters) + 64);
    // one run type per batch: TL ('C', 'S', 'I'), arrivals ('A', 'a'), arrivals and
    // eigen hits ('V', 'v') or eigen hits ('E')
    auto kind = [](char t) {
        return (t == 'A' || t == 'a') ? 1 : (t == 'V' || t == 'v') ? 4 : (t == 'E' ? 2 : (t == 'R' ? 3 : 0));
    };
    const int k0 = kind(r->envs[0].T.run_type[0]);
    r->arrivals = k0 == 1 || k0 == 4;
    r->also_eigen = k0 == 4;
    r->eigen = k0 == 2;
    r->rayrun = k0 == 3;
    r->raysets.assign(r->envs.size(), RaySet3{});
    r->nx2d = r->envs[0].T.nx2d;
    for(const auto &S : r->envs)
        if(S.T.nx2d != r->nx2d) throw std::runtime_error("a 3-D batch must be all 3-D or all Nx2D");
    auto rc = [](char b) { return b == 'g' || b == 'b'; };
    r->raycen = !r->rayrun && rc(r->envs[0].T.beam_type[0]);
    for(const auto &S : r->envs)
        if(!r->rayrun && rc(S.T.beam_type[0]) != r->raycen)
            throw std::runtime_error("a 3-D batch must use Cartesian or ray-centred beams throughout");
    for(const auto &S : r->envs)
        if(kind(S.T.run_type[0]) != k0) throw std::runtime_error("a 3-D batch must use one run type");
    auto bits = [](unsigned long long n) { int b = 1; while(b < 64 && (1ull << b) < n) ++b; return b; };
    if(r->rayrun) return;   // trajectories only: no segments, fields or arrivals
    // eigen-hit ordering key (low to high): depth | bearing | walk position |
    // step | ray | trace group; ray-centred beams walk depth, then bearing,
    // then the ranges: walk | bearing | depth
    auto eigen_layout = [&]() {
        int mz = 1, mt = 1, mr = 1, mj = 1;
        for(const auto &S : r->envs) {
            mz = std::max(mz, (int)S.T.rz.size());
            mt = std::max(mt, (int)S.T.theta.size());
            mr = std::max(mr, (int)S.T.rr.size());
        }
        for(const GroupDev &G : r->groups_h) mj = std::max(mj, G.njobs);
        ArrKeyBits kb{};
        kb.eigen = 1;
        const int lo = r->raycen ? mr : mz, hi = r->raycen ? mz : mr;
        kb.sh_theta = bits((unsigned long long)lo);
        kb.sh_walk = kb.sh_theta + bits((unsigned long long)mt);
        kb.sh_is = kb.sh_walk + bits((unsigned long long)hi);
        kb.sh_job = kb.sh_is + bits(100000);   // steps per ray (MaxN)
        kb.sh_cell = kb.sh_job + bits((unsigned long long)mj);
        kb.total_bits = kb.sh_cell + bits((unsigned long long)r->groups_h.size());
        if(kb.total_bits > 64) throw MemError("eigen-hit ordering key needs more than 64 bits; split the batch");
        return kb;
    };
    r->hits_h.clear();
    r->hit_group.clear();
    if(r->eigen) {
        r->kb = eigen_layout();
        return;
    }
    if(r->also_eigen) r->kb_eig = eigen_layout();
    if(!r->arrivals) {
        r->field.ensure(std::max<int64_t>(r->total_field, 1) * sizeof(float2));
        return;
    }
    // ordering key (low to high): step | ray | receiver cell
    int max_njobs = 1;
    for(const GroupDev &G : r->groups_h) max_njobs = std::max(max_njobs, G.njobs);
    ArrKeyBits kb{};
    kb.sh_is = 0;
    kb.sh_job = bits(100000);   // steps per ray (MaxN, include/bhc/structs.hpp:66)
    kb.sh_cell = kb.sh_job + bits((unsigned long long)max_njobs);
    kb.total_bits = kb.sh_cell + bits((unsigned long long)r->total_field);
    if(kb.total_bits > 64) throw MemError("arrival ordering key needs more than 64 bits; split the batch");
    r->kb = kb;
    const size_t cells = (size_t)r->total_field;
    int32_t mx = r->opt_max_narr;
    if(mx <= 0) {
        // as the reference (src/mode/arr.hpp:80-98): what a quarter of
        // max_memory holds per receiver, at most 1000
        uint64_t m = (r->max_memory / 4) / (cells * sizeof(ArrivalRec) + 1);
        if(r->also_eigen) m /= 2;   // half the room goes to the eigen hits (src/mode/arr.hpp:87)
        mx = (int32_t)std::min<uint64_t>(m, 1000);
    }
    if(mx <= 0) throw MemError("insufficient memory to allocate arrivals");
    r->max_narr = mx;
    r->narr_d.ensure(cells * sizeof(int32_t));
    r->arr_d.ensure(cells * (size_t)mx * sizeof(ArrivalRec));
    CK(cudaMemsetAsync(r->narr_d.p, 0, cells * sizeof(int32_t), st));
    h2d = A.bytes.size() + r->groups_h.size() * sizeof(GroupDev);
}

struct RangeStats {
    RunCounters rc{};
    double trace_ms = 0, infl_ms = 0;
};

// Arrivals of the traced jobs [j0, j1): candidates counted, written with
// their ordering keys, sorted, then replayed per receiver cell after the
// arrivals of earlier (lower-numbered) jobs. Returns false, having changed
// nothing, when the candidates do not fit in max_memory.
bool apply_arrivals(Run3 *r, long long j0, long long j1, unsigned long long nseg, cudaStream_t st, int sm_count,
                    RangeStats &acc)
{
    (void)j0; (void)j1;
    RunCounters *ctr = reinterpret_cast<RunCounters *>(r->counters.p);
    unsigned long long *cursor = reinterpret_cast<unsigned long long *>(
        reinterpret_cast<uint8_t *>(r->counters.p) + sizeof(RunCounters) + 8);
    const int igrid = sm_count * 8;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, st));
    // Nx2D: 2-D records on the bearing planes; 3-D: SegRec3
    auto gather = [&](bool count, ArrCand *c, uint64_t *k, uint32_t *v, unsigned long long cap,
                      unsigned long long *cur, const ArrKeyBits &kb) {
        if(r->raycen) {
            int nzt = 1;   // (depth, bearing) pairs per record, the most of the batch
            for(const auto &S : r->envs) nzt = std::max(nzt, (int)(S.T.rz.size() * S.T.theta.size()));
            return launch_arr_gather3d_rc((const XSeg3 *)r->segs.p, nseg, (const GroupDev *)r->groups_d.p,
                                          (int)r->groups_h.size(), count, c, k, v, cap, cur, ctr, kb, nzt,
                                          sm_count * 16, st);
        }
        return r->nx2d ? launch_arr_gather_nx(r->segs.p, nseg, (const GroupDev *)r->groups_d.p,
                                              (int)r->groups_h.size(), count, c, k, v, cap, cur, ctr, kb, igrid, st)
                       : launch_arr_gather3d((const SegRec3 *)r->segs.p, nseg, (const GroupDev *)r->groups_d.p,
                                             (int)r->groups_h.size(), count, c, k, v, cap, cur, ctr, kb, igrid, st);
    };
    // one pass: count, gather, order, then replay (AddArr) or emit the eigen
    // hits (RecordEigenHit); 'V' / 'v' runs take an eigen pass after the
    // arrivals pass, over the same segments
    unsigned long long n_first = 0;
    auto pass = [&](const ArrKeyBits &kb, bool eig, bool first) -> bool {
        CK(cudaMemsetAsync(&ctr->nevals, 0, sizeof(unsigned long long), st));
        CK(gather(true, nullptr, nullptr, nullptr, 0, nullptr, kb));
        unsigned long long n = 0;
        CK(cudaMemcpyAsync(&n, &ctr->nevals, sizeof n, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        const size_t per = sizeof(ArrCand) + 2 * sizeof(uint64_t) + 2 * sizeof(uint32_t);
        const size_t fixed = r->segs.bytes + r->arr_d.bytes + r->narr_d.bytes + (64u << 20);
        const size_t avail = r->max_memory > fixed ? r->max_memory - fixed : 0;
        if(first && (size_t)n * per + radix_sort_hist_entries(n) * 4 > avail && j1 - j0 > 1) return false;
        if(n > 0xffffffffull) throw MemError("more than 2^32 arrival candidates in one wave; lower max_memory");
        if(first) n_first = n;
        if(!n) return true;
        r->cand.ensure(n * sizeof(ArrCand));
        r->keys0.ensure(n * sizeof(uint64_t));
        r->keys1.ensure(n * sizeof(uint64_t));
        r->vals0.ensure(n * sizeof(uint32_t));
        r->vals1.ensure(n * sizeof(uint32_t));
        r->hist.ensure(std::max<size_t>(radix_sort_hist_entries(n), 1) * sizeof(uint32_t));
        CK(cudaMemsetAsync(cursor, 0, sizeof(unsigned long long), st));
        CK(gather(false, (ArrCand *)r->cand.p, (uint64_t *)r->keys0.p, (uint32_t *)r->vals0.p, n, cursor, kb));
        int in1 = 0;
        CK(radix_sort_pairs((uint64_t *)r->keys0.p, (uint32_t *)r->vals0.p, (uint64_t *)r->keys1.p,
                            (uint32_t *)r->vals1.p, n, kb.total_bits, (uint32_t *)r->hist.p, &in1, st));
        const uint64_t *k = (const uint64_t *)(in1 ? r->keys1.p : r->keys0.p);
        const uint32_t *v = (const uint32_t *)(in1 ? r->vals1.p : r->vals0.p);
        if(eig) {
            r->hits_d.ensure(n * sizeof(EigenHitRec));
            r->hitgrp_d.ensure(n * sizeof(int32_t));
            CK(launch_eigen_emit3(v, (const ArrCand *)r->cand.p, n, (const GroupDev *)r->groups_d.p,
                                  (int)r->groups_h.size(), (EigenHitRec *)r->hits_d.p, (int32_t *)r->hitgrp_d.p,
                                  sm_count, st));
            const size_t h0 = r->hits_h.size();
            r->hits_h.resize(h0 + n);
            r->hit_group.resize(h0 + n);
            CK(cudaMemcpyAsync(r->hits_h.data() + h0, r->hits_d.p, n * sizeof(EigenHitRec), cudaMemcpyDeviceToHost,
                               st));
            CK(cudaMemcpyAsync(r->hit_group.data() + h0, r->hitgrp_d.p, n * sizeof(int32_t),
                               cudaMemcpyDeviceToHost, st));
        } else {
            CK(launch_arr_replay(k, v, (const ArrCand *)r->cand.p, n, (const GroupDev *)r->groups_d.p,
                                 (int)r->groups_h.size(), nullptr, (long long)r->total_field, kb.sh_cell,
                                 r->max_narr, r->allow_merging, (int32_t *)r->narr_d.p, (ArrivalRec *)r->arr_d.p,
                                 sm_count, st, true));
        }
        return true;
    };
    if(!pass(r->kb, r->eigen, true)) {
        cudaEventDestroy(e0); cudaEventDestroy(e1);
        return false;
    }
    if(r->also_eigen) {
        CK(cudaStreamSynchronize(st));   // the replay reads the candidates the eigen pass rewrites
        pass(r->kb_eig, true, false);
    }
    const unsigned long long n = n_first;
    CK(cudaEventRecord(e1, st));
    RunCounters rc{};
    CK(cudaMemcpyAsync(&rc, ctr, sizeof rc, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    acc.rc.nevals += n;
    acc.rc.err_bits |= rc.err_bits;
    acc.rc.warn_bits |= rc.warn_bits;
    acc.infl_ms += ms;
    return true;
}

// trace the jobs [j0, j1) and apply their contributions; on a segment buffer
// overflow the range is split in halves (waves), which add into the same field
void run_jobs(Run3 *r, long long j0, long long j1, cudaStream_t st, int sm_count, uint64_t max_memory,
              RangeStats &acc)
{
    const size_t rec = r->nx2d ? nx_record_bytes() : (r->raycen ? sizeof(XSeg3) : sizeof(SegRec3));
    // TL: the field; arrivals: their storage, and half of the rest is left
    // for the arrival candidates
    const bool cand_mode = r->arrivals || r->eigen;
    const size_t fbytes = r->arrivals ? r->arr_d.bytes + r->narr_d.bytes
                                      : (r->eigen ? 0 : (size_t)r->total_field * sizeof(float2));
    size_t budget = max_memory > fbytes + (64u << 20) ? max_memory - fbytes - (64u << 20) : 0;
    if(cand_mode) budget /= 2;
    const unsigned long long maxcap = budget / rec;
    if(r->seg_cap == 0) {
        // a first guess within the budget: a ray emits at most one record per
        // step that brackets receiver ranges, about one per range it crosses
        // (plus the unused tail of its last 32-slot block)
        unsigned long long per_ray = 64;
        for(const auto &S : r->envs) {
            const Env3Tables &T = S.T;
            const double steps = 2.0 * std::max(T.box_x, T.box_y) / std::max(T.deltas, 1e-9);
            per_ray = std::max<unsigned long long>(
                per_ray, (unsigned long long)std::min<double>(steps, 1.1 * T.rr.size()) + 32);
        }
        r->seg_cap = std::min<unsigned long long>(maxcap, std::max<unsigned long long>(1u << 16, per_ray * (j1 - j0)));
    }
    for(int attempt = 0; attempt < 6; ++attempt) {
        if(r->seg_cap < 1024) throw MemError("max_memory leaves no room for 3-D segment records");
        r->segs.ensure(r->seg_cap * rec);
        RunCounters *ctr = reinterpret_cast<RunCounters *>(r->counters.p);
        unsigned long long *jc = reinterpret_cast<unsigned long long *>(
            reinterpret_cast<uint8_t *>(r->counters.p) + sizeof(RunCounters));
        RunCounters zero{};
        zero.overflow_job = 0xffffffffu;
        CK(cudaMemcpyAsync(ctr, &zero, sizeof zero, cudaMemcpyHostToDevice, st));
        unsigned long long j0u = (unsigned long long)j0;
        CK(cudaMemcpyAsync(jc, &j0u, sizeof j0u, cudaMemcpyHostToDevice, st));
        cudaEvent_t e0, e1, e2;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        CK(cudaEventCreate(&e2));
        CK(cudaEventRecord(e0, st));
        const long long nj = j1 - j0;
        const int tgrid = (int)std::max<long long>(1, std::min<long long>((nj + 63) / 64, (long long)sm_count * 16));
        if(r->nx2d)
            CK(launch_trace_nx((const GroupDev *)r->groups_d.p, (int)r->groups_h.size(), j1, r->segs.p, r->seg_cap,
                               ctr, jc, tgrid, st));
        else if(r->raycen)
            CK(launch_trace3d_rc((const GroupDev *)r->groups_d.p, (int)r->groups_h.size(), j1, (XSeg3 *)r->segs.p,
                                 r->seg_cap, ctr, jc, tgrid, st));
        else
            CK(launch_trace3d((const GroupDev *)r->groups_d.p, (int)r->groups_h.size(), j1, (SegRec3 *)r->segs.p,
                              r->seg_cap, ctr, jc, tgrid, st));
        CK(cudaEventRecord(e1, st));
        RunCounters rc{};
        CK(cudaMemcpyAsync(&rc, ctr, sizeof rc, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        float tms = 0;
        CK(cudaEventElapsedTime(&tms, e0, e1));
        if(rc.err_bits & (1u << ERR_SEG_OVERFLOW)) {
            cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2);
            if(r->seg_cap < maxcap) {
                r->seg_cap = std::min<unsigned long long>(maxcap, std::max(r->seg_cap * 2, (unsigned long long)(rc.nseg * 1.25)));
                continue;
            }
            if(nj <= 1) throw MemError("one ray's segments exceed max_memory; raise bhcb_init.max_memory");
            const long long mid = j0 + nj / 2;
            run_jobs(r, j0, mid, st, sm_count, max_memory, acc);
            run_jobs(r, mid, j1, st, sm_count, max_memory, acc);
            return;
        }
        const unsigned long long nseg = std::min(rc.nseg, r->seg_cap);
        const int igrid = sm_count * 8;
        if(cand_mode && rc.err_bits == 0) {
            cudaEventDestroy(e0); cudaEventDestroy(e2);
            if(!apply_arrivals(r, j0, j1, nseg, st, sm_count, acc)) {   // candidates exceed the budget
                cudaEventDestroy(e1);
                const long long mid = j0 + nj / 2;
                run_jobs(r, j0, mid, st, sm_count, max_memory, acc);
                run_jobs(r, mid, j1, st, sm_count, max_memory, acc);
                return;
            }
            cudaEventDestroy(e1);
            acc.rc.nseg += nseg;
            acc.rc.nsteps += rc.nsteps;
            acc.rc.warn_bits |= rc.warn_bits;
            acc.trace_ms += tms;
            return;
        }
        if(rc.err_bits == 0 && r->nx2d) {
            int nz = 1;
            for(const auto &S : r->envs) nz = std::max(nz, (int)S.T.rz.size());
            CK(launch_influence_nx(r->segs.p, nseg, (const GroupDev *)r->groups_d.p, (int)r->groups_h.size(),
                                   (float2 *)r->field.p, ctr, nz, sm_count * 16, st));
        } else if(rc.err_bits == 0 && r->raycen) {
            int nzt = 1;   // (depth, bearing) pairs per record, the most of the batch
            for(const auto &S : r->envs) nzt = std::max(nzt, (int)(S.T.rz.size() * S.T.theta.size()));
            CK(launch_influence3d_rc((const XSeg3 *)r->segs.p, nseg, (const GroupDev *)r->groups_d.p,
                                     (int)r->groups_h.size(), (float2 *)r->field.p, ctr, nzt, sm_count * 16, st));
        } else if(rc.err_bits == 0) {
            CK(launch_influence3d((const SegRec3 *)r->segs.p, nseg, (const GroupDev *)r->groups_d.p,
                                  (int)r->groups_h.size(), (float2 *)r->field.p, ctr, igrid, st, r->mixed));
        }
        CK(cudaEventRecord(e2, st));
        RunCounters rc2{};
        CK(cudaMemcpyAsync(&rc2, ctr, sizeof rc2, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        float ims = 0;
        CK(cudaEventElapsedTime(&ims, e1, e2));
        cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2);
        acc.rc.nseg += nseg;
        acc.rc.nsteps += rc2.nsteps;
        acc.rc.nevals += rc2.nevals;
        acc.rc.err_bits |= rc2.err_bits;
        acc.rc.warn_bits |= rc2.warn_bits;
        acc.trace_ms += tms;
        acc.infl_ms += ims;
        return;
    }
    throw MemError("3-D segment buffer overflow persisted");
}

} // namespace

namespace {
// take-off declination (deg) of the local ray index of environment S
// (GetJobIndices, src/common.hpp:365-391: ialpha fastest)
double alpha_deg_of(const Env3Tables &T, int local)
{
    const int ialpha = T.isingle_alpha >= 1 ? T.isingle_alpha - 1 : local % (int)T.alpha.size();
    return (180.0 / M_PI) * T.alpha[ialpha];
}

// Trajectories of R.jobs (limits as for the ray kernel): a count pass sizes the
// point buffer exactly, a second pass of the same deterministic trace writes
// the points. Returns the tracer's error bits.
uint32_t trace_rays3(Run3 *r, RaySet3 &R, cudaStream_t st, uint32_t &warn_bits)
{
    const int n = (int)R.jobs.size();
    R.npts.assign(n, 0);
    R.bnc.assign(2 * (size_t)n, 0);
    R.off.assign(n, 0);
    R.xyz.clear();
    R.valid = true;
    if(n == 0) return 0;
    DevBuf jobs_d, lim_d, npts_d, bnc_d, off_d, pts_d;
    jobs_d.ensure(n * sizeof(long long));
    lim_d.ensure(n * sizeof(int));
    npts_d.ensure(n * sizeof(int));
    bnc_d.ensure(2 * (size_t)n * sizeof(int));
    off_d.ensure(n * sizeof(long long));
    RunCounters *ctr = (RunCounters *)r->counters.p;
    const GroupDev *G = (const GroupDev *)r->groups_d.p;
    const int ng = (int)r->groups_h.size();
    CK(cudaMemcpyAsync(jobs_d.p, R.jobs.data(), n * sizeof(long long), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(lim_d.p, R.limits.data(), n * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(ctr, 0, sizeof(RunCounters), st));
    auto rays = r->nx2d ? launch_rays_nx : launch_rays3d;   // Nx2D: 2-D rays, points in ocean coordinates
    CK(rays(G, ng, (const long long *)jobs_d.p, (const int *)lim_d.p, n, nullptr, nullptr, (int *)npts_d.p,
                     (int *)bnc_d.p, ctr, true, r->sm_count, st));
    CK(cudaMemcpyAsync(R.npts.data(), npts_d.p, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(R.bnc.data(), bnc_d.p, 2 * (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, st));
    RunCounters rc{};
    CK(cudaMemcpyAsync(&rc, ctr, sizeof rc, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    warn_bits |= rc.warn_bits;
    if(rc.err_bits) return rc.err_bits;
    long long tot = 0;
    for(int i = 0; i < n; ++i) {
        R.off[i] = tot;
        tot += R.npts[i];
    }
    if((uint64_t)tot * 3 * sizeof(double) > r->max_memory) throw MemError("ray points exceed max_memory");
    pts_d.ensure(std::max<long long>(tot, 1) * 3 * sizeof(double));
    CK(cudaMemcpyAsync(off_d.p, R.off.data(), n * sizeof(long long), cudaMemcpyHostToDevice, st));
    CK(rays(G, ng, (const long long *)jobs_d.p, (const int *)lim_d.p, n, (const long long *)off_d.p,
                     (double *)pts_d.p, (int *)npts_d.p, (int *)bnc_d.p, ctr, false, r->sm_count, st));
    R.xyz.resize(3 * (size_t)tot);
    if(tot) CK(cudaMemcpyAsync(R.xyz.data(), pts_d.p, tot * 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return 0;
}
} // namespace

uint32_t run3_run(Run3 *r, cudaStream_t st, int sm_count, uint64_t max_memory, int32_t opt_max_narr,
                  int32_t allow_merging, bool mixed, bhcb_stats &stats, uint32_t &warn_bits)
{
    auto t0 = std::chrono::steady_clock::now();
    uint64_t h2d = 0;
    r->mixed = mixed;
    r->max_memory = max_memory;
    r->opt_max_narr = opt_max_narr;
    r->allow_merging = allow_merging;
    r->sm_count = sm_count;
    prepare3(r, st, h2d);
    if(r->rayrun) {   // RunRayMode (src/mode/ray.cpp:163-198): every ray of every environment
        stats = bhcb_stats{};
        warn_bits = 0;
        uint32_t eb = 0;
        for(size_t i = 0; i < r->envs.size() && !eb; ++i) {
            const GroupDev &G = r->groups_h[i];
            RaySet3 &R = r->raysets[i];
            R = RaySet3{};
            for(int local = 0; local < G.njobs; ++local) {
                R.jobs.push_back(G.job_base + local);
                R.limits.push_back(-1);
                R.alpha_deg.push_back(alpha_deg_of(r->envs[i].T, local));
            }
            eb = trace_rays3(r, R, st, warn_bits);
        }
        r->ran = eb == 0;
        stats.rays = (uint64_t)r->njobs;
        stats.groups = stats.fields = (int32_t)r->envs.size();
        stats.err_bits = eb;
        stats.warn_bits = warn_bits;
        stats.h2d_bytes = h2d;
        stats.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return eb;
    }
    const bool tl = !r->arrivals && !r->eigen;
    if(tl) CK(cudaMemsetAsync(r->field.p, 0, std::max<int64_t>(r->total_field, 1) * sizeof(float2), st));
    RangeStats acc;
    run_jobs(r, 0, r->njobs, st, sm_count, max_memory, acc);
    if(acc.rc.err_bits == 0 && tl) {
        for(size_t i = 0; i < r->envs.size(); ++i) {
            const auto &S = r->envs[i];
            if(r->nx2d)   // 2-D pressure scaling along each plane's ranges
                CK(launch_scale_nx((float2 *)r->field.p, (const GroupDev *)r->groups_d.p, (int)i, sm_count * 4, st));
            else if(S.T.run_type[0] != 'C')
                CK(launch_sqrt3d((float2 *)r->field.p + S.field_base, S.field_n, sm_count * 4, st));
        }
        CK(cudaStreamSynchronize(st));
    }
    r->ran = acc.rc.err_bits == 0;
    stats = bhcb_stats{};
    stats.rays = (uint64_t)r->njobs;
    stats.steps = acc.rc.nsteps;
    stats.segments = acc.rc.nseg;
    stats.evals = acc.rc.nevals;
    stats.err_bits = acc.rc.err_bits;
    stats.warn_bits = acc.rc.warn_bits;
    stats.groups = (int32_t)r->envs.size();
    stats.fields = (int32_t)r->envs.size();
    stats.trace_ms = acc.trace_ms;
    stats.influence_ms = acc.infl_ms;
    stats.influence_span_ms = acc.infl_ms;
    stats.h2d_bytes = h2d;
    stats.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    warn_bits = acc.rc.warn_bits;
    return acc.rc.err_bits;
}

void run3_shape(const Run3 *r, int env, int32_t dims[6])
{
    if(env < 0 || env >= (int)r->envs.size()) throw std::invalid_argument("env_index out of range");
    const Env3Tables &T = r->envs[env].T;
    dims[0] = (int32_t)T.sz.size();
    dims[1] = (int32_t)T.sx.size();
    dims[2] = (int32_t)T.sy.size();
    dims[3] = (int32_t)T.theta.size();
    dims[4] = (int32_t)T.rz.size();
    dims[5] = (int32_t)T.rr.size();
}

static const Env3Slot &ran_env(const Run3 *r, int env)
{
    if(env < 0 || env >= (int)r->envs.size()) throw std::invalid_argument("env_index out of range");
    if(!r->ran) throw StateError("no completed 3-D run: call bhcb_run first");
    return r->envs[env];
}

void run3_copy_field(Run3 *r, int env, void *dst, size_t bytes, cudaStream_t st)
{
    const Env3Slot &S = ran_env(r, env);
    if(r->arrivals || r->eigen || r->rayrun)
        throw StateError("not a TL run: use bhcb_copy_arrivals / bhcb_eigen_hits / bhcb_copy_rays");
    const size_t need = (size_t)S.field_n * sizeof(float2);
    if(!dst || bytes < need) throw std::invalid_argument("destination too small");
    CK(cudaMemcpyAsync(dst, (float2 *)r->field.p + S.field_base, need, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
}

void *run3_field_device(Run3 *r, int env)
{
    const Env3Slot &S = ran_env(r, env);
    if(r->arrivals || r->eigen || r->rayrun) throw StateError("not a TL run");
    return (float2 *)r->field.p + S.field_base;
}

void run3_grid(const Run3 *r, int env, std::vector<double> &sx, std::vector<double> &sy, std::vector<float> &sz,
               std::vector<double> &rr, std::vector<float> &rz, std::vector<double> &theta)
{
    if(env < 0 || env >= (int)r->envs.size()) throw std::invalid_argument("env_index out of range");
    const Env3Tables &T = r->envs[env].T;
    sx = T.sx; sy = T.sy; sz = T.sz; rr = T.rr; rz = T.rz; theta = T.theta;
}

std::vector<std::string> run3_warnings(const Run3 *r, int env)
{
    if(env < 0 || env >= (int)r->envs.size()) throw std::invalid_argument("env_index out of range");
    return r->envs[env].T.warnings;
}

bool run3_is_arrivals(const Run3 *r) { return r->arrivals; }

int64_t run3_eigen_hits(Run3 *r, int env, void *hits, int64_t max_hits)
{
    ran_env(r, env);
    if(!r->eigen && !r->also_eigen) throw StateError("not an eigen-hit run");
    int64_t n = 0;
    EigenHitRec *out = reinterpret_cast<EigenHitRec *>(hits);
    for(size_t k = 0; k < r->hits_h.size(); ++k) {
        if(r->hit_group[k] != env) continue;
        if(out && n < max_hits) out[n] = r->hits_h[k];
        ++n;
    }
    return n;
}

int32_t run3_max_narr(const Run3 *r) { return r->max_narr; }

void run3_copy_arrivals(Run3 *r, int env, int32_t *narr, size_t narr_bytes, void *arr, size_t arr_bytes,
                        cudaStream_t st)
{
    const Env3Slot &S = ran_env(r, env);
    if(!r->arrivals) throw StateError("not an arrivals run");
    const size_t cells = (size_t)S.field_n;
    if(narr) {
        if(narr_bytes < cells * sizeof(int32_t)) throw std::invalid_argument("narr buffer too small");
        CK(cudaMemcpyAsync(narr, (int32_t *)r->narr_d.p + S.field_base, cells * sizeof(int32_t),
                           cudaMemcpyDeviceToHost, st));
    }
    if(arr) {
        const size_t need = cells * (size_t)r->max_narr * sizeof(ArrivalRec);
        if(arr_bytes < need) throw std::invalid_argument("arrival buffer too small");
        CK(cudaMemcpyAsync(arr, (ArrivalRec *)r->arr_d.p + (size_t)S.field_base * r->max_narr, need,
                           cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
}

// WriteOutArrivals, 3-D (src/mode/arr.cpp:88-239): binary for RunType 'a',
// list-directed text for 'A'
static void write_arrivals3(Run3 *r, const Env3Slot &S, const std::string &path, cudaStream_t st)
{
    const Env3Tables &T = S.T;
    const size_t cells = (size_t)S.field_n;
    std::vector<int32_t> narr(cells);
    std::vector<ArrivalRec> arr(cells * (size_t)r->max_narr);
    run3_copy_arrivals(r, (int)(&S - r->envs.data()), narr.data(), narr.size() * 4, arr.data(),
                       arr.size() * sizeof(ArrivalRec), st);
    const double RadDeg = 180.0 / 3.14159265358979323846;
    const bool ascii = T.run_type[0] == 'A' || T.run_type[0] == 'V';   // src/mode/arr.cpp:95-100
    std::ofstream o(path, std::ios::binary);
    if(!o.good()) throw std::runtime_error("cannot open " + path);
    const int nsx = (int)T.sx.size(), nsy = (int)T.sy.size(), nsz = (int)T.sz.size();
    const int nth = (int)T.theta.size(), nrz = (int)T.rz.size(), nrr = (int)T.rr.size();
    char b[256];
    if(ascii) {
        o << "3D\n";
        snprintf(b, sizeof b, "%.9g\n", T.freq0);
        o << b;
        o << nsx; for(double v : T.sx) { snprintf(b, sizeof b, " %.17g", v); o << b; } o << "\n";
        o << nsy; for(double v : T.sy) { snprintf(b, sizeof b, " %.17g", v); o << b; } o << "\n";
        o << nsz; for(float v : T.sz) { snprintf(b, sizeof b, " %.9g", v); o << b; } o << "\n";
        o << nrz; for(float v : T.rz) { snprintf(b, sizeof b, " %.9g", v); o << b; } o << "\n";
        o << nrr; for(double v : T.rr) { snprintf(b, sizeof b, " %.17g", v); o << b; } o << "\n";
        o << nth; for(double v : T.theta) { snprintf(b, sizeof b, " %.17g", v); o << b; } o << "\n";
    } else {
        RecWriter w(o);
        w.put_bytes("'3D'", 4); w.end();
        w.put((float)T.freq0); w.end();
        w.put((int32_t)nsx); w.put_bytes(T.sx.data(), T.sx.size() * 8); w.end();
        w.put((int32_t)nsy); w.put_bytes(T.sy.data(), T.sy.size() * 8); w.end();
        w.put((int32_t)nsz); w.put_bytes(T.sz.data(), T.sz.size() * 4); w.end();
        w.put((int32_t)nrz); w.put_bytes(T.rz.data(), T.rz.size() * 4); w.end();
        w.put((int32_t)nrr); w.put_bytes(T.rr.data(), T.rr.size() * 8); w.end();
        w.put((int32_t)nth); w.put_bytes(T.theta.data(), T.theta.size() * 8); w.end();
    }
    RecWriter w(o);
    const size_t per_src = (size_t)nth * nrz * nrr;
    for(int isz = 0; isz < nsz; ++isz)
        for(int isx = 0; isx < nsx; ++isx)
            for(int isy = 0; isy < nsy; ++isy) {
                const size_t cb = (((size_t)isz * nsx + isx) * nsy + isy) * per_src;
                int32_t maxn = 0;   // MaxNPerSource (src/mode/arr.cpp:24-74)
                for(size_t k = 0; k < per_src; ++k) maxn = std::max(maxn, narr[cb + k]);
                if(ascii) o << maxn << "\n";
                else { w.put(maxn); w.end(); }
                for(size_t k = 0; k < per_src; ++k) {
                    const size_t base = cb + k;
                    const int32_t n = narr[base];
                    if(ascii) o << n << "\n";
                    else { w.put(n); w.end(); }
                    for(int a = 0; a < n; ++a) {
                        const ArrivalRec &A = arr[base * r->max_narr + a];
                        if(ascii) {
                            snprintf(b, sizeof b, "%.9g %.17g %.9g %.9g %.9g %.9g %.9g %.9g %d %d\n", A.a,
                                     RadDeg * A.Phase, A.delay_re, A.delay_im, A.SrcDeclAngle, A.SrcAzimAngle,
                                     A.RcvrDeclAngle, A.RcvrAzimAngle, A.NTopBnc, A.NBotBnc);
                            o << b;
                        } else {
                            w.put(A.a);
                            w.put((float)(RadDeg * A.Phase));
                            w.put(A.delay_re);
                            w.put(A.delay_im);
                            w.put(A.SrcDeclAngle);
                            w.put(A.SrcAzimAngle);
                            w.put(A.RcvrDeclAngle);
                            w.put(A.RcvrAzimAngle);
                            w.put((float)A.NTopBnc);
                            w.put((float)A.NBotBnc);
                            w.end();
                        }
                    }
                }
            }
}

// .shd, 3-D: WriteHeader and WriteOutTL (src/mode/tl.cpp:38-101, 195-248)
bool run3_has_rays(const Run3 *r) { return r->rayrun || r->eigen || r->also_eigen; }

// RunType 'R': the traced rays; 'E', 'V', 'v': the hit rays re-traced up to their hit
// (EigenModePostWorker, src/mode/eigen.cpp:24-45) on first use, in hit order
static const RaySet3 &rays_of_env(Run3 *r, int env, cudaStream_t st)
{
    const Env3Slot &S = ran_env(r, env);
    if(!r->rayrun && !r->eigen && !r->also_eigen)
        throw StateError("rays exist for ray runs ('R') and eigen runs ('E', 'V', 'v')");
    RaySet3 &R = r->raysets[env];
    if(R.valid) return R;
    if(r->rayrun) throw StateError("no rays: run first");
    const Env3Tables &T = S.T;
    const GroupDev &G = r->groups_h[env];
    const int nal = T.isingle_alpha >= 1 ? 1 : (int)T.alpha.size();
    const int nbe = T.isingle_beta >= 1 ? 1 : (int)T.beta.size();
    const int nsx = (int)T.sx.size(), nsy = (int)T.sy.size();
    for(size_t k = 0; k < r->hits_h.size(); ++k) {
        if(r->hit_group[k] != env) continue;
        const EigenHitRec &h = r->hits_h[k];
        const int ia = T.isingle_alpha >= 1 ? 0 : h.ialpha;
        const int ib = T.isingle_beta >= 1 ? 0 : h.ibeta;
        const long long local = ((((long long)h.isz * nsx + h.isx) * nsy + h.isy) * nbe + ib) * nal + ia;
        R.jobs.push_back(G.job_base + local);
        R.limits.push_back(h.is);
        R.alpha_deg.push_back((180.0 / M_PI) * T.alpha[h.ialpha]);
    }
    uint32_t wb = 0;
    const uint32_t eb = trace_rays3(r, R, st, wb);
    if(eb) {
        R.valid = false;
        char b[96];
        snprintf(b, sizeof b, "tracer error bits 0x%x while re-tracing eigenrays", eb);
        throw std::runtime_error(b);
    }
    return R;
}

void run3_rays_shape(Run3 *r, int env, cudaStream_t st, int64_t &nrays, int64_t &npoints)
{
    const RaySet3 &R = rays_of_env(r, env, st);
    nrays = (int64_t)R.jobs.size();
    npoints = (int64_t)(R.xyz.size() / 3);
}

void run3_copy_rays(Run3 *r, int env, cudaStream_t st, int32_t *npts, int32_t *bounces, double *alpha_deg,
                    double *xyz, size_t xyz_bytes)
{
    const RaySet3 &R = rays_of_env(r, env, st);
    if(xyz && xyz_bytes < R.xyz.size() * sizeof(double)) throw std::invalid_argument("point buffer too small");
    if(npts) std::memcpy(npts, R.npts.data(), R.npts.size() * sizeof(int32_t));
    if(bounces) std::memcpy(bounces, R.bnc.data(), R.bnc.size() * sizeof(int32_t));
    if(alpha_deg) std::memcpy(alpha_deg, R.alpha_deg.data(), R.alpha_deg.size() * sizeof(double));
    if(xyz && !R.xyz.empty()) std::memcpy(xyz, R.xyz.data(), R.xyz.size() * sizeof(double));
}

// .ray file, 3-D (OpenRAYFile / WriteRay, src/mode/ray.hpp:176-247): take-off
// angles in radians, points (x, y, z)
static void write_rays3(Run3 *r, int env, const std::string &path, cudaStream_t st)
{
    const Env3Slot &S = r->envs[env];
    const RaySet3 &R = rays_of_env(r, env, st);
    const Env3Tables &T = S.T;
    std::ofstream o(path);
    if(!o.good()) throw std::runtime_error("cannot open " + path);
    char b[160];
    o << "'" << S.in.title << "'\n";
    snprintf(b, sizeof b, "%.17g\n", T.freq0);
    o << b;
    o << T.sx.size() << " " << T.sy.size() << " " << T.sz.size() << "\n";
    o << T.alpha.size() << " " << T.beta.size() << "\n";
    snprintf(b, sizeof b, "%.17g\n%.17g\n", S.in.ssp_z.empty() ? 0.0 : S.in.ssp_z[0], S.in.bot_depth);
    o << b;
    o << "'xyz'\n";
    for(size_t i = 0; i < R.jobs.size(); ++i) {
        if(R.npts[i] <= 0) continue;
        snprintf(b, sizeof b, "%.17g\n", R.alpha_deg[i] * (M_PI / 180.0));
        o << b;
        o << R.npts[i] << " " << R.bnc[2 * i] << " " << R.bnc[2 * i + 1] << "\n";
        for(int k = 0; k < R.npts[i]; ++k) {
            const double *q = &R.xyz[3 * (R.off[i] + k)];
            snprintf(b, sizeof b, "%.17g %.17g %.17g\n", q[0], q[1], q[2]);
            o << b;
        }
    }
}

void run3_writeout(Run3 *r, int env, const std::string &root, cudaStream_t st)
{
    const Env3Slot &S = ran_env(r, env);
    if(r->eigen || r->rayrun) {
        write_rays3(r, env, root + ".ray", st);
        return;
    }
    if(r->arrivals) {
        write_arrivals3(r, S, root + ".arr", st);
        if(r->also_eigen) write_rays3(r, env, root + ".ray", st);   // src/api.cpp:465-486
        return;
    }
    const Env3Tables &T = S.T;
    std::vector<float2> u((size_t)S.field_n);
    CK(cudaMemcpyAsync(u.data(), (float2 *)r->field.p + S.field_base, u.size() * sizeof(float2),
                       cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const int nsx = (int)T.sx.size(), nsy = (int)T.sy.size(), nsz = (int)T.sz.size();
    const int nth = (int)T.theta.size(), nrz = (int)T.rz.size(), nrr = (int)T.rr.size();
    int32_t lrecl = 84;
    lrecl = std::max<int32_t>(lrecl, 2 * 1 * 8);
    lrecl = std::max<int32_t>(lrecl, nth * 8);
    lrecl = std::max<int32_t>(lrecl, nsx * 8);
    lrecl = std::max<int32_t>(lrecl, nsy * 8);
    lrecl = std::max<int32_t>(lrecl, nsz * 4);
    lrecl = std::max<int32_t>(lrecl, nrz * 4);
    lrecl = std::max<int32_t>(lrecl, nrr * 8);
    const size_t nrec = 10 + (size_t)nsx * nsy * nth * nsz * nrz;
    std::vector<uint8_t> buf((size_t)lrecl * nrec, 0);
    auto rec = [&](size_t k) { return buf.data() + k * lrecl; };
    int32_t lw = lrecl / 4;
    std::memcpy(rec(0), &lw, 4);
    std::string title = S.in.title;
    title.resize(80, ' ');
    std::memcpy(rec(0) + 4, title.data(), 80);
    std::memcpy(rec(1), "rectilin  ", 10);
    const int32_t hdr[7] = {1, nth, nsx, nsy, nsz, nrz, nrr};
    std::memcpy(rec(2), hdr, sizeof hdr);
    const double f0 = T.freq0, atten = 0.0;
    std::memcpy(rec(2) + 28, &f0, 8);
    std::memcpy(rec(2) + 36, &atten, 8);
    std::memcpy(rec(3), &f0, 8);
    std::memcpy(rec(4), T.theta.data(), (size_t)nth * 8);
    std::memcpy(rec(5), T.sx.data(), (size_t)nsx * 8);
    std::memcpy(rec(6), T.sy.data(), (size_t)nsy * 8);
    std::memcpy(rec(7), T.sz.data(), (size_t)nsz * 4);
    std::memcpy(rec(8), T.rz.data(), (size_t)nrz * 4);
    std::memcpy(rec(9), T.rr.data(), (size_t)nrr * 8);
    for(int isx = 0; isx < nsx; ++isx)
        for(int isy = 0; isy < nsy; ++isy)
            for(int it = 0; it < nth; ++it)
                for(int isz = 0; isz < nsz; ++isz)
                    for(int iz = 0; iz < nrz; ++iz) {
                        const size_t k = 10 + ((((size_t)isx * nsy + isy) * nth + it) * nsz + isz) * nrz + iz;
                        const size_t a = (((((size_t)isz * nsx + isx) * nsy + isy) * nth + it) * nrz + iz) * nrr;
                        std::memcpy(rec(k), &u[a], (size_t)nrr * 8);
                    }
    std::ofstream o(root + ".shd", std::ios::binary);
    if(!o.good()) throw std::runtime_error("cannot open " + root + ".shd");
    o.write((const char *)buf.data(), buf.size());
}

} // namespace bhcb
