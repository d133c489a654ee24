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

cudaError_t launch_trace3d(const GroupDev *, int, long long, SegRec3 *, unsigned long long, RunCounters *,
                           unsigned long long *, int, cudaStream_t);
cudaError_t launch_influence3d(const SegRec3 *, unsigned long long, const GroupDev *, int, float2 *, RunCounters *,
                               int, cudaStream_t);
cudaError_t launch_sqrt3d(float2 *, long long, int, cudaStream_t);

namespace {
struct Env3Slot {
    std::string root;
    EnvInput in;
    Env3Tables T;
    int64_t field_base = 0, field_n = 0;
};
} // namespace

struct Run3 {
    std::vector<Env3Slot> envs;
    std::vector<GroupDev> groups_h;
    DevBuf arena, groups_d, segs, counters, field;
    long long njobs = 0;
    unsigned long long seg_cap = 0;
    int64_t total_field = 0;
    bool ran = false;
};

Run3 *run3_new() { return new Run3(); }

void run3_free(Run3 *r)
{
    if(!r) return;
    for(DevBuf *b : {&r->arena, &r->groups_d, &r->segs, &r->counters, &r->field}) b->release();
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
                  alpha, beta, sbp; };
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
        offs.push_back(o);

        Env3Dev d{};
        EnvDev &e = d.e1d;
        e.ssp_type = T.ssp_type == SSP_HEXAHEDRAL ? SSP_CLINEAR : T.ssp_type;
        e.nssp = (int)T.z.size();
        e.top = T.top;
        e.bot = T.bot;
        e.freq0 = T.freq0;
        e.deltas = T.deltas;
        d.hex = T.ssp_type == SSP_HEXAHEDRAL;
        d.hnx = (int)T.hx.size(); d.hny = (int)T.hy.size(); d.hnz = (int)T.hz.size();
        d.top = T.top;
        d.bot = T.bot;
        d.top_nx = T.top_nx; d.top_ny = T.top_ny; d.bot_nx = T.bot_nx; d.bot_ny = T.bot_ny;
        d.nsx = (int)T.sx.size(); d.nsy = (int)T.sy.size(); d.nsz = (int)T.sz.size();
        d.nrr = (int)T.rr.size(); d.nrz = (int)T.rz.size(); d.ntheta = (int)T.theta.size();
        d.nalpha = (int)T.alpha.size(); d.nbeta = (int)T.beta.size();
        d.isingle_alpha = T.isingle_alpha; d.isingle_beta = T.isingle_beta;
        d.dalpha = T.dalpha; d.dbeta = T.dbeta; d.deltas = T.deltas;
        d.box_x = T.box_x; d.box_y = T.box_y; d.box_z = T.box_z; d.freq0 = T.freq0;
        d.gaussian = T.beam_type[0] == 'B';
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
        d.hx = dptr<double>(ab, o.hx); d.hy = dptr<double>(ab, o.hy); d.hz = dptr<double>(ab, o.hz);
        d.hc = dptr<double>(ab, o.hc); d.hcz = dptr<double>(ab, o.hcz);
        d.btop = dptr<Bdry3PtDev>(ab, o.btop); d.bbot = dptr<Bdry3PtDev>(ab, o.bbot);
        d.sx = dptr<double>(ab, o.sx); d.sy = dptr<double>(ab, o.sy); d.sz = dptr<float>(ab, o.sz);
        d.rr = dptr<double>(ab, o.rr); d.rz = dptr<float>(ab, o.rz); d.tcs = dptr<double>(ab, o.tcs);
        d.alpha = dptr<double>(ab, o.alpha); d.beta = dptr<double>(ab, o.beta); d.sbp = dptr<double>(ab, o.sbp);
        r->groups_h[i].env3 = dptr<Env3Dev>(ab, env_off + i * sizeof(Env3Dev));
    }
    CK(cudaMemcpyAsync(ab, A.bytes.data(), A.bytes.size(), cudaMemcpyHostToDevice, st));
    r->groups_d.ensure(r->groups_h.size() * sizeof(GroupDev));
    CK(cudaMemcpyAsync(r->groups_d.p, r->groups_h.data(), r->groups_h.size() * sizeof(GroupDev),
                       cudaMemcpyHostToDevice, st));
    r->field.ensure(std::max<int64_t>(r->total_field, 1) * sizeof(float2));
    r->counters.ensure(sizeof(RunCounters) + 64);
    h2d = A.bytes.size() + r->groups_h.size() * sizeof(GroupDev);
}

struct RangeStats {
    RunCounters rc{};
    double trace_ms = 0, infl_ms = 0;
};

// trace the jobs [j0, j1) and apply their contributions; on a segment buffer
// overflow the range is split in halves (waves), which add into the same field
void run_jobs(Run3 *r, long long j0, long long j1, cudaStream_t st, int sm_count, uint64_t max_memory,
              RangeStats &acc)
{
    const size_t rec = sizeof(SegRec3);
    const size_t fbytes = (size_t)r->total_field * sizeof(float2);
    const size_t budget = max_memory > fbytes + (64u << 20) ? max_memory - fbytes - (64u << 20) : 0;
    const unsigned long long maxcap = budget / rec;
    if(r->seg_cap == 0) {
        // a first guess: 64 records per ray, within the budget
        r->seg_cap = std::min<unsigned long long>(maxcap, std::max<unsigned long long>(1u << 16, 64ull * (j1 - j0)));
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
        if(rc.err_bits == 0)
            CK(launch_influence3d((const SegRec3 *)r->segs.p, nseg, (const GroupDev *)r->groups_d.p,
                                  (int)r->groups_h.size(), (float2 *)r->field.p, ctr, igrid, st));
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

uint32_t run3_run(Run3 *r, cudaStream_t st, int sm_count, uint64_t max_memory, bhcb_stats &stats, uint32_t &warn_bits)
{
    auto t0 = std::chrono::steady_clock::now();
    uint64_t h2d = 0;
    prepare3(r, st, h2d);
    CK(cudaMemsetAsync(r->field.p, 0, std::max<int64_t>(r->total_field, 1) * sizeof(float2), st));
    RangeStats acc;
    run_jobs(r, 0, r->njobs, st, sm_count, max_memory, acc);
    if(acc.rc.err_bits == 0) {
        for(const auto &S : r->envs)
            if(S.T.run_type[0] != 'C')
                CK(launch_sqrt3d((float2 *)r->field.p + S.field_base, S.field_n, sm_count * 4, st));
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
    const size_t need = (size_t)S.field_n * sizeof(float2);
    if(!dst || bytes < need) throw std::invalid_argument("destination too small");
    CK(cudaMemcpyAsync(dst, (float2 *)r->field.p + S.field_base, need, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
}

void *run3_field_device(Run3 *r, int env)
{
    const Env3Slot &S = ran_env(r, env);
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

// .shd, 3-D: WriteHeader and WriteOutTL (src/mode/tl.cpp:38-101, 195-248)
void run3_writeout(Run3 *r, int env, const std::string &root, cudaStream_t st)
{
    const Env3Slot &S = ran_env(r, env);
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
