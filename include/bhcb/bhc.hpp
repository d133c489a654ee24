/*
 * bhc:: drop-in surface of the B200 beam tracer (libbhcb.so).
 *
 * The same public interface as the reference's include/bhc/bhc.hpp:58-452
 * and include/bhc/structs.hpp:490-572 (bhcInit, bhcParams, bhcOutputs and the
 * structures their members point to, with the same member names and meaning),
 * so that a program written against the reference's library builds against
 * this header and links libbhcb.so instead. Implemented in C++ over the C ABI
 * of include/bhcb.h (bellhopcuda_b200/csrc/host/bhc_cxx.cpp).
 *
 * Differences a caller can see:
 *   - real is double (the reference's default build); SSP arrays are
 *     allocated with room for MaxSSP nodes, as the reference's fixed arrays.
 *   - 2-D runs take their parameters from bhcParams in memory (after setup
 *     from a file or from the defaults, and any extsetup_* / edits). 3-D and
 *     Nx2D runs read FileRoot's files: bhcParams<true> reports the setup's
 *     values, edits to it are not used by run.
 *   - outputs.rayinfo holds each ray's points (x) and bounce counts; the other
 *     rayPt members are zero.
 *   - readout reads .shd (TL) files.
 *   - the tracer is the FP64 one unless BHCB_PRECISION=mixed is set in the
 *     environment.
 * Functions return false on failure and report the reason through
 * bhcInit::outputCallback (stdout when it is null), as the reference does.
 */
#pragma once
#include <complex>
#include <cstddef>
#include <cstdint>
#include <type_traits>

namespace bhc {

using real = double;
using cpx = std::complex<real>;
using cpxf = std::complex<float>;

struct vec2 {
    real x, y;
};
struct vec3 {
    real x, y, z;
};
struct int2 {
    int32_t x, y;
};
template<bool X3D> using VEC23 = typename std::conditional<X3D, vec3, vec2>::type;
template<bool X3D> using IORI2 = typename std::conditional<X3D, int2, int32_t>::type;

constexpr int32_t MaxN = 100000;
constexpr int32_t MaxSSP = MaxN + 1;
constexpr int32_t MaxBioLayers = 200;

struct rxyz_vector {
    real *r, *x, *y, *z;
};

struct SSPStructure {
    real *z, *rho;                   // MaxSSP nodes each
    real *alphaR, *alphaI, *betaR, *betaI;
    real *cMat, *czMat;              // quad: c[iz * Nr + ir]; hexahedral: c[(ix * Ny + iy) * Nz + iz]
    rxyz_vector Seg;                 // quad / hexahedral profile coordinates
    int32_t NPts, Nr, Nx, Ny, Nz;
    char Type;
    char AttenUnit[2];
    bool rangeInKm;
    bool dirty;
};

struct HSInfo {
    real alphaR, betaR, alphaI, betaI;
    cpx cP, cS;
    real rho, Depth;
    char bc;
    char Opt[6];
};
struct HSExtra {
    real zTemp, Mz;
    real Sigma;
};
struct BdryPtSmall {
    HSInfo hs;
    HSExtra hsx;
};
struct BdryType {
    BdryPtSmall Top, Bot;
};

template<bool O3D> struct BdryPtFull {
    VEC23<O3D> x;                    // 2-D: (range, depth) of the node
    VEC23<O3D> t, n;
    HSInfo hs;                       // 2-D long format: the segment's halfspace
};
template<bool O3D> struct BdryInfoTopBot {
    IORI2<O3D> NPts;
    char type[2];
    bool dirty;
    bool rangeInKm;
    BdryPtFull<O3D> *bd;
    int32_t NBotProvinces;
    HSInfo *BotProv;
};
template<bool O3D> struct BdryInfo {
    BdryInfoTopBot<O3D> top, bot;
};

struct ReflectionCoef {
    real theta, r, phi;
};
struct ReflectionInfoTopBot {
    int32_t NPts;
    bool inDegrees;
    ReflectionCoef *r;
};
struct ReflectionInfo {
    ReflectionInfoTopBot bot, top;
};

struct bioStructure {
    real z1, z2, f0, q, a0;
};
struct AttenInfo {
    int32_t NBioLayers;
    bioStructure bio[MaxBioLayers];
    real t, Salinity, pH, z_bar, fg;
    int32_t NMedia;
};

struct Position {
    int32_t NSx, NSy, NSz, NRz, NRr, Ntheta;
    int32_t NRz_per_range;
    bool SxSyInKm, RrInKm;
    bool thetaDuplRemoved;
    real Delta_r, Delta_theta;
    real *Sx, *Sy;
    float *Sz;
    real *Rr;
    float *Rz;
    real *theta;
    vec2 *t_rcvr;
};

struct AngleInfo {
    int32_t n, iSingle;
    real d;
    real *angles;
    bool inDegrees;
};
struct AnglesStructure {
    AngleInfo alpha, beta;
};

struct FreqInfo {
    real freq0;
    int32_t Nfreq;
    real *freqVec;
};

template<bool O3D> struct BeamStructure {
    int32_t NBeams, Nimage, iBeamWindow;
    char Component;
    char Type[4];
    char RunType[7];
    bool rangeInKm;
    bool autoDeltas;
    real deltas, epsMultiplier, rLoop;
    VEC23<O3D> Box;
};

struct SBPInfo {
    char SBPFlag;
    bool SBPIndB;
    int32_t NSBPPts;
    real *SrcBmPat;
};

struct EigenHit {
    int32_t is;
    int32_t itheta, ir, iz;
    int32_t isx, isy, isz, ialpha, ibeta;
};
struct EigenInfo {
    int32_t neigen;
    int32_t memsize;
    EigenHit *hits;
};

struct Arrival {
    int32_t NTopBnc, NBotBnc;
    float SrcDeclAngle, SrcAzimAngle, RcvrDeclAngle, RcvrAzimAngle, a, Phase;
    cpxf delay;
};
struct ArrInfo {
    Arrival *Arr;
    int32_t *NArr;
    int32_t *MaxNPerSource;
    int32_t MaxNArr;
    bool AllowMerging;
};

template<bool R3D> struct rayPt {
    int32_t NumTopBnc, NumBotBnc;
    VEC23<R3D> x;
    VEC23<R3D> t;
    real c;
    real Amp, Phase;
    cpx tau;
};
template<bool O3D, bool R3D> struct RayResult {
    rayPt<R3D> *ray;
    real SrcDeclAngle;
    int32_t Nsteps;
};
template<bool O3D, bool R3D> struct RayInfo {
    RayResult<O3D, R3D> *results;
    int32_t NRays;
};

struct bhcInit {
    int32_t numThreads = -1;
    size_t maxMemory = 4ull * 1024ull * 1024ull * 1024ull;
    bool useRayCopyMode = false;
    int gpuIndex = 0;
    const char *FileRoot = nullptr;
    void (*prtCallback)(const char *message) = nullptr;
    void (*outputCallback)(const char *message) = nullptr;
    void (*completedCallback)() = nullptr;
};

template<bool O3D> struct bhcParams {
    char Title[80];
    real fT;
    BdryType *Bdry;
    BdryInfo<O3D> *bdinfo;
    ReflectionInfo *refl;
    SSPStructure *ssp;
    AttenInfo *atten;
    Position *Pos;
    AnglesStructure *Angles;
    FreqInfo *freqinfo;
    BeamStructure<O3D> *Beam;
    SBPInfo *sbp;
    void *internal;
};

template<bool O3D, bool R3D> struct bhcOutputs {
    RayInfo<O3D, R3D> *rayinfo;
    cpxf *uAllSources;
    EigenInfo *eigen;
    ArrInfo *arrinfo;
};

template<bool O3D, bool R3D> bool setup(const bhcInit &init, bhcParams<O3D> &params, bhcOutputs<O3D, R3D> &outputs);
template<bool O3D> void extsetup_sxsy(bhcParams<O3D> &params, int32_t NSx, int32_t NSy);
template<bool O3D> void extsetup_sz(bhcParams<O3D> &params, int32_t NSz);
template<bool O3D> void extsetup_rcvrranges(bhcParams<O3D> &params, int32_t NRr);
template<bool O3D> void extsetup_rcvrdepths(bhcParams<O3D> &params, int32_t NRz);
template<bool O3D> void extsetup_rcvrbearings(bhcParams<O3D> &params, int32_t Ntheta);
template<bool O3D> void extsetup_rayelevations(bhcParams<O3D> &params, int32_t n);
template<bool O3D> void extsetup_raybearings(bhcParams<O3D> &params, int32_t n);
template<bool O3D> void extsetup_sbp(bhcParams<O3D> &params, int32_t NSBPPts);
template<bool O3D> void extsetup_freqvec(bhcParams<O3D> &params, int32_t Nfreq);
template<bool O3D> void extsetup_altimetry(bhcParams<O3D> &params, const IORI2<O3D> &NPts);
template<bool O3D> void extsetup_bathymetry(bhcParams<O3D> &params, const IORI2<O3D> &NPts,
                                            const int32_t &NBotProvinces);
template<bool O3D> void extsetup_trc(bhcParams<O3D> &params, int32_t NPts);
template<bool O3D> void extsetup_brc(bhcParams<O3D> &params, int32_t NPts);
void extsetup_ssp_quad(bhcParams<false> &params, int32_t NPts, int32_t Nr);
void extsetup_ssp_hexahedral(bhcParams<true> &params, int32_t Nx, int32_t Ny, int32_t Nz);
template<bool O3D> void extsetup_blocking(bhcParams<O3D> &params, const bool &blocking);
template<bool O3D> bool echo(bhcParams<O3D> &params);
template<bool O3D, bool R3D> bool run(bhcParams<O3D> &params, bhcOutputs<O3D, R3D> &outputs);
template<bool O3D, bool R3D> bool postprocess(bhcParams<O3D> &params, bhcOutputs<O3D, R3D> &outputs);
template<bool O3D> int get_percent_progress(bhcParams<O3D> &params);
template<bool O3D, bool R3D> bool writeout(const bhcParams<O3D> &params, const bhcOutputs<O3D, R3D> &outputs,
                                           const char *FileRoot);
template<bool O3D, bool R3D> bool readout(bhcParams<O3D> &params, bhcOutputs<O3D, R3D> &outputs,
                                          const char *FileRoot);
template<bool O3D> bool writeenv(bhcParams<O3D> &params, const char *FileRoot);
template<bool O3D, bool R3D> void finalize(bhcParams<O3D> &params, bhcOutputs<O3D, R3D> &outputs);
template<bool O3D, bool R3D> bool get_ssp(bhcParams<O3D> &params, const VEC23<R3D> &x, float &sound_speed);

// explicit instantiations exported by libbhcb.so (2-D, Nx2D, 3-D)
#define BHCB_DIMS(M) M(false, false) M(true, false) M(true, true)
#define BHCB_EXTERN_RUN(O, R)                                                                              \
    extern template bool setup<O, R>(const bhcInit &, bhcParams<O> &, bhcOutputs<O, R> &);               \
    extern template bool run<O, R>(bhcParams<O> &, bhcOutputs<O, R> &);                                   \
    extern template bool postprocess<O, R>(bhcParams<O> &, bhcOutputs<O, R> &);                           \
    extern template bool writeout<O, R>(const bhcParams<O> &, const bhcOutputs<O, R> &, const char *);    \
    extern template bool readout<O, R>(bhcParams<O> &, bhcOutputs<O, R> &, const char *);                 \
    extern template void finalize<O, R>(bhcParams<O> &, bhcOutputs<O, R> &);                              \
    extern template bool get_ssp<O, R>(bhcParams<O> &, const VEC23<R> &, float &);
BHCB_DIMS(BHCB_EXTERN_RUN)
#undef BHCB_EXTERN_RUN
#undef BHCB_DIMS

} // namespace bhc
