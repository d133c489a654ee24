// A program written against the bhc:: interface (include/bhcb/bhc.hpp), built
// and run by tests/test_bhc_api.py and tests/test_gpu_bhc_api.py.
//
//   bhc_api_check params <dir>
//       setup from the defaults and from files, extsetup_* resizing, writeenv
//       round trip, get_ssp, echo; needs no GPU.
//   bhc_api_check run <file root | -> <field.bin> [<writeout root>]
//       setup (from FileRoot, or the defaults for "-"), run, write the field
//       [NSz][NRz_per_range][NRr] complex float to field.bin; with a writeout
//       root also writeout and readout, and check the read field is the same.
//   bhc_api_check nonblocking <file root>
//       extsetup_blocking(false): run returns at once, postprocess waits,
//       completedCallback fires once, progress ends at 100.
//   bhc_api_check writeenv <2|3|4> <file root> <new root>
//       setup from the files, writeenv to the new root, setup from those;
//       the two setups agree. Needs no GPU.
//   bhc_api_check ssp <3|4> <file root> <x y z | r z>
//       get_ssp of a 3-D or Nx2D setup at one point; needs no GPU.
//   bhc_api_check run3arr <file root>
//       a 3-D arrivals run through bhc::run; counts and MaxNPerSource.
//   bhc_api_check readout <2|3|4> <file root>
//       setup from the files (2-D, 3-D or Nx2D) and readout of the run's
//       output file (.arr for RunType 'A' / 'a', .ray for 'R'); prints the
//       counts and sums the test compares with its own reading of the file;
//       needs no GPU.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "bhcb/bhc.hpp"

static int failures = 0;
#define EXPECT(c)                                                                                           \
    do {                                                                                                    \
        if(!(c)) {                                                                                          \
            std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c);                                        \
            ++failures;                                                                                     \
        }                                                                                                   \
    } while(0)

static std::atomic<int> completed{0};
static void on_output(const char *m) { std::printf("out: %s\n", m); }
static void on_print(const char *m) { std::printf("%s", m); }
static void on_done() { ++completed; }

static bhc::bhcInit make_init(const char *root)
{
    bhc::bhcInit init;
    init.FileRoot = root;
    init.outputCallback = on_output;
    init.prtCallback = on_print;
    init.completedCallback = on_done;
    return init;
}

static void same_params(const bhc::bhcParams<false> &a, const bhc::bhcParams<false> &b)
{
    EXPECT(std::strncmp(a.Title, b.Title, 80) == 0);
    EXPECT(a.freqinfo->freq0 == b.freqinfo->freq0);
    EXPECT(a.ssp->NPts == b.ssp->NPts);
    for(int i = 0; i < a.ssp->NPts && i < b.ssp->NPts; ++i) {
        EXPECT(a.ssp->z[i] == b.ssp->z[i]);
        EXPECT(a.ssp->alphaR[i] == b.ssp->alphaR[i]);
    }
    EXPECT(a.Bdry->Bot.hs.Depth == b.Bdry->Bot.hs.Depth);
    EXPECT(std::memcmp(a.Bdry->Top.hs.Opt, b.Bdry->Top.hs.Opt, 4) == 0);
    EXPECT(a.Bdry->Bot.hs.bc == b.Bdry->Bot.hs.bc);
    EXPECT(a.Pos->NSz == b.Pos->NSz && a.Pos->NRz == b.Pos->NRz && a.Pos->NRr == b.Pos->NRr);
    for(int i = 0; i < a.Pos->NSz && i < b.Pos->NSz; ++i) EXPECT(a.Pos->Sz[i] == b.Pos->Sz[i]);
    for(int i = 0; i < a.Pos->NRz && i < b.Pos->NRz; ++i) EXPECT(a.Pos->Rz[i] == b.Pos->Rz[i]);
    for(int i = 0; i < a.Pos->NRr && i < b.Pos->NRr; ++i) EXPECT(a.Pos->Rr[i] == b.Pos->Rr[i]);
    EXPECT(a.Angles->alpha.n == b.Angles->alpha.n);
    for(int i = 0; i < a.Angles->alpha.n && i < b.Angles->alpha.n; ++i)
        EXPECT(a.Angles->alpha.angles[i] == b.Angles->alpha.angles[i]);
    EXPECT(std::memcmp(a.Beam->RunType, b.Beam->RunType, 5) == 0);
    EXPECT(a.Beam->Box.x == b.Beam->Box.x && a.Beam->Box.y == b.Beam->Box.y);
    EXPECT(a.bdinfo->bot.NPts == b.bdinfo->bot.NPts);
    for(int i = 0; i < a.bdinfo->bot.NPts && i < b.bdinfo->bot.NPts; ++i) {
        EXPECT(a.bdinfo->bot.bd[i].x.x == b.bdinfo->bot.bd[i].x.x);
        EXPECT(a.bdinfo->bot.bd[i].x.y == b.bdinfo->bot.bd[i].x.y);
    }
}

static int check_params(const std::string &dir)
{
    using namespace bhc;
    bhcParams<false> p;
    bhcOutputs<false, false> o;
    EXPECT(setup(make_init(nullptr), p, o));
    // the modules' defaults
    EXPECT(std::strcmp(p.Title, "no env file") == 0);
    EXPECT(p.freqinfo->freq0 == 50.0);
    EXPECT(p.Pos->NSz == 1 && std::fabs(p.Pos->Sz[0] - 567.8f) < 1e-3f);
    EXPECT(p.Pos->NRz == 11 && p.Pos->Rz[10] == 5000.0f);
    EXPECT(p.Pos->NRr == 10 && p.Pos->Rr[9] == 50.0);
    EXPECT(p.Angles->alpha.n > 2);
    EXPECT(p.Angles->alpha.angles[0] == -20.0 && p.Angles->alpha.angles[p.Angles->alpha.n - 1] == 20.0);
    EXPECT(std::memcmp(p.Beam->RunType, "CG RR", 5) == 0);
    EXPECT(p.Bdry->Bot.hs.Depth == 5000.0);
    float c = 0;
    EXPECT((get_ssp<false, false>(p, vec2{1000.0, 100.0}, c)));
    EXPECT(c == 1500.0f);
    EXPECT(echo(p));
    // writeenv round trip
    const std::string r1 = dir + "/defaults";
    EXPECT(writeenv(p, r1.c_str()));
    bhcParams<false> q;
    bhcOutputs<false, false> qo;
    EXPECT(setup(make_init(r1.c_str()), q, qo));
    same_params(p, q);
    // edits: more ranges, a bathymetry, a downward-refracting profile
    extsetup_rcvrranges(q, 20);
    for(int i = 0; i < 20; ++i) q.Pos->Rr[i] = 2.5 * (i + 1);
    extsetup_bathymetry(q, 3, 0);
    q.bdinfo->bot.type[0] = 'L';
    q.bdinfo->bot.type[1] = 'S';
    const double br[3] = {0.0, 25.0, 60.0}, bz[3] = {5000.0, 4000.0, 4500.0};
    for(int i = 0; i < 3; ++i) q.bdinfo->bot.bd[i].x = vec2{br[i], bz[i]};
    q.ssp->alphaR[1] = 1480.0;
    const std::string r2 = dir + "/edited";
    EXPECT(writeenv(q, r2.c_str()));
    bhcParams<false> e;
    bhcOutputs<false, false> eo;
    EXPECT(setup(make_init(r2.c_str()), e, eo));
    same_params(q, e);
    EXPECT(e.Pos->NRr == 20 && e.Pos->Rr[19] == 50.0);
    EXPECT(e.bdinfo->bot.NPts == 3);
    float c1 = 0;
    EXPECT((get_ssp<false, false>(e, vec2{0.0, 5000.0}, c1)));
    EXPECT(std::fabs(c1 - 1480.0f) < 1e-3f);
    EXPECT((get_ssp<false, false>(e, vec2{0.0, 2500.0}, c1)));
    EXPECT(std::fabs(c1 - 1490.0f) < 1e-3f);   // 'C' linear between the nodes
    // a missing file is reported, not thrown
    bhcParams<false> m;
    bhcOutputs<false, false> mo;
    EXPECT(!setup(make_init((dir + "/missing").c_str()), m, mo));
    finalize(m, mo);
    finalize(e, eo);
    finalize(q, qo);
    finalize(p, o);
    std::printf(failures ? "FAILED %d\n" : "OK\n", failures);
    return failures ? 1 : 0;
}

static bool write_field(const char *path, const bhc::cpxf *u, size_t n)
{
    FILE *f = std::fopen(path, "wb");
    if(!f) return false;
    const bool ok = std::fwrite(u, sizeof(bhc::cpxf), n, f) == n;
    std::fclose(f);
    return ok;
}

static int check_run(const char *root, const char *out, const char *wroot)
{
    using namespace bhc;
    bhcParams<false> p;
    bhcOutputs<false, false> o;
    const bool from_file = std::strcmp(root, "-") != 0;
    if(!setup(make_init(from_file ? root : nullptr), p, o)) return 2;
    if(!run(p, o)) return 3;
    EXPECT(completed == 1);
    EXPECT(get_percent_progress(p) == 100);
    const size_t n = (size_t)p.Pos->NSz * p.Pos->NRz_per_range * p.Pos->NRr;
    EXPECT(o.uAllSources != nullptr);
    if(o.uAllSources && !write_field(out, o.uAllSources, n)) return 4;
    if(wroot) {
        EXPECT(writeout(p, o, wroot));
        bhcParams<false> r;
        bhcOutputs<false, false> ro;
        EXPECT(setup(make_init(nullptr), r, ro));
        EXPECT(readout(r, ro, wroot));
        EXPECT(r.Pos->NRr == p.Pos->NRr && r.Pos->NSz == p.Pos->NSz);
        if(ro.uAllSources && o.uAllSources) EXPECT(std::memcmp(ro.uAllSources, o.uAllSources, n * 8) == 0);
        finalize(r, ro);
    }
    finalize(p, o);
    std::printf(failures ? "FAILED %d\n" : "OK\n", failures);
    return failures ? 1 : 0;
}

static int check_nonblocking(const char *root)
{
    using namespace bhc;
    bhcParams<false> p;
    bhcOutputs<false, false> o;
    if(!setup(make_init(root), p, o)) return 2;
    extsetup_blocking(p, false);
    EXPECT(run(p, o));
    int last = -1;
    for(int i = 0; i < 100000 && completed == 0; ++i) last = get_percent_progress(p);
    EXPECT(postprocess(p, o));
    EXPECT(completed == 1);
    EXPECT(get_percent_progress(p) == 100);
    EXPECT(o.uAllSources != nullptr);
    (void)last;
    finalize(p, o);
    std::printf(failures ? "FAILED %d\n" : "OK\n", failures);
    return failures ? 1 : 0;
}

template<bool O3D, bool R3D> static int check_readout(const char *root)
{
    using namespace bhc;
    bhcParams<O3D> p;
    bhcOutputs<O3D, R3D> o;
    if(!setup(make_init(root), p, o)) return 2;
    if(!readout(p, o, root)) {
        finalize(p, o);
        return 3;
    }
    const char run0 = p.Beam->RunType[0];
    if(run0 == 'A' || run0 == 'a') {
        const ArrInfo &A = *o.arrinfo;
        const Position &P = *p.Pos;
        const size_t cells = (size_t)P.NSx * P.NSy * P.NSz * P.Ntheta * P.NRz * P.NRr;
        double s[10] = {0};
        long long total = 0;
        for(size_t c = 0; c < cells; ++c)
            for(int k = 0; k < A.NArr[c]; ++k) {
                const Arrival &r = A.Arr[c * A.MaxNArr + k];
                ++total;
                s[0] += r.a; s[1] += r.Phase; s[2] += r.delay.real(); s[3] += r.delay.imag();
                s[4] += r.SrcDeclAngle; s[5] += r.SrcAzimAngle; s[6] += r.RcvrDeclAngle; s[7] += r.RcvrAzimAngle;
                s[8] += r.NTopBnc; s[9] += r.NBotBnc;
            }
        int maxsrc = 0;
        for(int k = 0; k < P.NSx * P.NSy * P.NSz; ++k) maxsrc = std::max(maxsrc, A.MaxNPerSource[k]);
        std::printf("arr %d %d %d %d %d %d %.9g %lld %d %d", P.NSx, P.NSy, P.NSz, P.Ntheta, P.NRz, P.NRr,
                    (double)p.freqinfo->freq0, total, A.MaxNArr, maxsrc);
        for(double v : s) std::printf(" %.17g", v);
        std::printf("\n");
    } else if(run0 == 'R') {
        const RayInfo<O3D, R3D> &R = *o.rayinfo;
        long long pts = 0;
        double s[6] = {0};
        for(int i = 0; i < R.NRays; ++i) {
            const RayResult<O3D, R3D> &r = R.results[i];
            pts += r.Nsteps;
            s[0] += r.SrcDeclAngle;
            for(int k = 0; k < r.Nsteps; ++k) {
                s[1] += r.ray[k].x.x;
                s[2] += r.ray[k].x.y;
                if constexpr(R3D) s[3] += r.ray[k].x.z;
            }
            s[4] += r.ray[r.Nsteps - 1].NumTopBnc;
            s[5] += r.ray[r.Nsteps - 1].NumBotBnc;
        }
        std::printf("ray %d %lld", R.NRays, pts);
        for(double v : s) std::printf(" %.17g", v);
        std::printf("\n");
    }
    finalize(p, o);
    std::printf(failures ? "FAILED %d\n" : "OK\n", failures);
    return failures ? 1 : 0;
}

template<bool O3D, bool R3D> static int check_writeenv(const char *root, const char *newroot)
{
    using namespace bhc;
    bhcParams<O3D> p;
    bhcOutputs<O3D, R3D> o;
    if(!setup(make_init(root), p, o)) return 2;
    EXPECT(writeenv(p, newroot));
    bhcParams<O3D> q;
    bhcOutputs<O3D, R3D> qo;
    EXPECT(setup(make_init(newroot), q, qo));
    EXPECT(std::strncmp(p.Title, q.Title, 80) == 0);
    EXPECT(p.Pos->NSz == q.Pos->NSz && p.Pos->NRz == q.Pos->NRz && p.Pos->NRr == q.Pos->NRr);
    EXPECT(p.Pos->Ntheta == q.Pos->Ntheta && p.Beam->RunType[0] == q.Beam->RunType[0]);
    finalize(q, qo);
    finalize(p, o);
    // without a prtCallback the PRT text goes to FileRoot.prt
    bhcInit quiet = make_init(newroot);
    quiet.prtCallback = nullptr;
    bhcParams<O3D> r;
    bhcOutputs<O3D, R3D> ro;
    EXPECT(setup(quiet, r, ro));
    EXPECT(echo(r));
    finalize(r, ro);
    FILE *f = std::fopen((std::string(newroot) + ".prt").c_str(), "r");
    EXPECT(f != nullptr);
    if(f) {
        char line[256] = {0};
        EXPECT(std::fgets(line, sizeof line, f) != nullptr);
        EXPECT(std::strstr(line, "bhcb (B200)") != nullptr);
        std::fclose(f);
    }
    std::printf(failures ? "FAILED %d\n" : "OK\n", failures);
    return failures ? 1 : 0;
}

// get_ssp of a 3-D (dim 3: x y z) or Nx2D (dim 4: r z) setup; prints c
template<bool O3D, bool R3D> static int check_ssp(const char *root, int argc, char **argv)
{
    using namespace bhc;
    bhcParams<O3D> p;
    bhcOutputs<O3D, R3D> o;
    if(!setup(make_init(root), p, o)) return 2;
    VEC23<R3D> x{};
    if constexpr(R3D) x = vec3{std::atof(argv[0]), std::atof(argv[1]), std::atof(argv[2])};
    else x = vec2{std::atof(argv[0]), std::atof(argv[1])};
    (void)argc;
    float c = -1.f;
    const bool ok = get_ssp<O3D, R3D>(p, x, c);
    std::printf("ssp %d %.9g\n", ok ? 1 : 0, (double)c);
    finalize(p, o);
    return ok ? 0 : 5;
}

// 3-D arrivals through bhc::run: the counts, their sum and MaxNPerSource
static int check_run3_arrivals(const char *root)
{
    using namespace bhc;
    bhcParams<true> p;
    bhcOutputs<true, true> o;
    bhcInit init = make_init(root);
    init.numThreads = 1;   // single-threaded: arrivals merge, as in the reference's fixture run
    if(!setup(init, p, o)) return 2;
    if(!run(p, o)) return 3;
    const Position &P = *p.Pos;
    const size_t nsrc = (size_t)P.NSx * P.NSy * P.NSz, per = (size_t)P.Ntheta * P.NRz * P.NRr;
    long long total = 0;
    for(size_t s = 0; s < nsrc; ++s) {
        int m = 0;
        for(size_t k = 0; k < per; ++k) {
            total += o.arrinfo->NArr[s * per + k];
            m = std::max(m, o.arrinfo->NArr[s * per + k]);
        }
        EXPECT(o.arrinfo->MaxNPerSource[s] == m);
        EXPECT(m <= o.arrinfo->MaxNArr);
    }
    std::printf("arr3 %zu %lld\n", nsrc, total);
    finalize(p, o);
    std::printf(failures ? "FAILED %d\n" : "OK\n", failures);
    return failures ? 1 : 0;
}

int main(int argc, char **argv)
{
    if(argc >= 3 && std::strcmp(argv[1], "run3arr") == 0) return check_run3_arrivals(argv[2]);
    if(argc >= 6 && std::strcmp(argv[1], "ssp") == 0) {
        const int d = std::atoi(argv[2]);
        if(d == 3 && argc >= 7) return check_ssp<true, true>(argv[3], argc - 4, argv + 4);
        if(d == 4) return check_ssp<true, false>(argv[3], argc - 4, argv + 4);
        return 64;
    }
    if(argc >= 5 && std::strcmp(argv[1], "writeenv") == 0) {
        const int d = std::atoi(argv[2]);
        return d == 3 ? check_writeenv<true, true>(argv[3], argv[4])
                      : d == 4 ? check_writeenv<true, false>(argv[3], argv[4])
                               : check_writeenv<false, false>(argv[3], argv[4]);
    }
    if(argc >= 4 && std::strcmp(argv[1], "readout") == 0) {
        const int d = std::atoi(argv[2]);
        return d == 3 ? check_readout<true, true>(argv[3]) : d == 4 ? check_readout<true, false>(argv[3])
                                                                    : check_readout<false, false>(argv[3]);
    }
    if(argc >= 3 && std::strcmp(argv[1], "params") == 0) return check_params(argv[2]);
    if(argc >= 4 && std::strcmp(argv[1], "run") == 0) return check_run(argv[2], argv[3], argc >= 5 ? argv[4] : nullptr);
    if(argc >= 3 && std::strcmp(argv[1], "nonblocking") == 0) return check_nonblocking(argv[2]);
    std::printf("usage: bhc_api_check params <dir> | run <root|-> <field.bin> [wroot] | nonblocking <root>\n");
    return 64;
}
