// Internal data layout shared by the host runtime and the sm_100a kernels.
//
// One "environment" (EnvDev) is the preprocessed, device-resident form of one
// bhcParams set (reference: include/bhc/structs.hpp:548-563) for one trace
// frequency. A "group" is one environment plus the list of frequencies whose
// fields are evaluated from its trajectories (1 for a plain run; N when the
// environment's tables are frequency independent and frequencies share one
// trajectory). A launch processes a batch of groups; its rays ("jobs") are
// numbered group-major, then source depth, then launch angle, matching the
// reference's job order within a group (src/common.hpp:347-391).
#pragma once
#include <stdint.h>

namespace bhcb {

// SSP interpolation types (reference: src/runtype.hpp:52-75)
enum SspType : int32_t { SSP_N2LINEAR = 0, SSP_CLINEAR = 1, SSP_CUBIC = 2, SSP_PCHIP = 3,
                         SSP_ANALYTIC = 4, SSP_HEXAHEDRAL = 5, SSP_QUAD = 6 };

// error / warning bits: same numbering as the reference's ErrState
// (src/util/errors.hpp:61-93); BHCB_ERR_SEG_OVERFLOW is this runtime's own.
enum : uint32_t {
    ERR_RAYINIT = 2, ERR_BOUNDARY_SEG_NAN = 3, ERR_BOUNDARY_CONDITION_TYPE = 4,
    ERR_INVALID_SSP_TYPE = 5, ERR_OUTSIDE_ALTIMETRY = 6, ERR_OUTSIDE_BATHYMETRY = 7,
    ERR_OUTSIDE_SSP = 8, ERR_QUAD_ISEG = 9,
    ERR_STAGE_WAIT = 30,             // a shared-memory table staging wait ran out (this runtime's own)
    ERR_SEG_OVERFLOW = 31,
};
enum : uint32_t {
    WARN_ONERAY_OUTOFMEMORY = 1, WARN_TOO_FEW_BEAMS = 3, WARN_SOURCE_OUTSIDE_BOUNDARIES = 4,
    WARN_UNBOUNDED_BEAM = 2, WARN_OUTSIDE_REFLCOEF = 5, WARN_CERVENY_WIDTH_BUGGY = 12,
    WARN_INVALID_WIDTH_BUGGY = 13,
    WARN_OUTSIDE_ALTIMETRY = 6, WARN_OUTSIDE_BATHYMETRY = 7,
    WARN_STEP_NEGATIVE_H = 8, WARN_TRIDIAG_H_NEGATIVE = 9, WARN_TRIDIAG_H_GROWING = 10,
    WARN_CPCHIP_INVALIDXT = 16, WARN_CPCHIP_INVALIDCCOEF = 17, WARN_OCEANTORAYX_GAVEUP = 18,
};

struct HsDev {          // halfspace (include/bhc/structs.hpp:93-101)
    double cPr, cPi, cSr, cSi, rho;
    int32_t bc;         // 'V','R','A','G'
    int32_t pad;
};

struct BdryPtDev {      // 2-D boundary node (include/bhc/structs.hpp:147-170)
    double x[2], t[2], n[2], Noden[2], Nodet[2];
    double Len, kappa;
    double cPr, cPi, cSr, cSi, rho;   // per-segment halfspace (long format 'L')
};

struct EnvDev {
    // SSP tables (reference SSPStructure, include/bhc/structs.hpp:73-91)
    int32_t ssp_type, nssp;
    const double *z, *rho;
    const double *c, *cz;      // complex, interleaved re/im, [nssp]
    const double *n2, *n2z;    // complex [nssp]
    const double *coef;        // complex [4][nssp]: spline (S) or pchip (P) coefficients
    // quad (range-dependent) SSP (src/ssp.hpp:157-212): profile ranges qr[nqr]
    // (m), sound speed qc[iz * nqr + ir] and its depth gradient qcz[iz * nqr + ir]
    int32_t nqr, pad_q;
    const double *qr, *qc, *qcz;
    // tabulated reflection coefficients for 'F' boundaries (src/module/reflcoef.hpp):
    // (theta deg, |R|, phase rad) triples, strictly increasing theta
    int32_t ntrc, nbrc;
    const double *trc, *brc;
    int32_t beam_shift;              // Beam->Type[3] == 'S' (src/reflect.hpp:383-448)
    // influence type other than geometric Cartesian (INFL_*), and the Cerveny
    // beam parameters (src/module/beaminfo.hpp:79-90)
    int32_t infl_kind;
    int32_t beam1;                   // Beam->Type[1]: width 'F', 'M', 'W' or 'C'
    int32_t nimage, ibeam_window, component;
    double eps_mult, rloop;
    double top_depth, bot_depth;     // Bdry->Top / Bot.hs.Depth (Cerveny images)
    HsDev top, bot;
    // boundaries
    int32_t ntop, nbot;
    int32_t top_curv, bot_curv;      // type[0] == 'C'
    int32_t top_long, bot_long;      // type[1] == 'L'
    const BdryPtDev *btop, *bbot;
    // receivers / sources / angles (include/bhc/structs.hpp:278-321)
    int32_t nrr, nrz, nrz_per_range, nsz, nalpha, isingle;
    const double *rr;
    const float *rz, *sz;
    const double *alpha;
    const double *acs;               // (cos, sin) pairs of alpha from the host's libm, as the reference's RayInit has them
    double dalpha, delta_r;
    // beam (include/bhc/structs.hpp:331-341)
    double deltas, box_x, box_y, freq0;
    int32_t run0;                    // RunType[0]
    int32_t beam0;                   // Beam->Type[0] after MoveBeamType
    int32_t beam2;                   // Beam->Type[2] curvature option
    int32_t gaussian, coherent, line_source, irregular, q_zero_init;
    // source beam pattern: pairs (angle deg, linear level)
    int32_t nsbp;
    int32_t arrivals;                // RunType 'A' / 'a': segments carry the receiver angle
    const double *sbp;
};

// 3-D grid boundary node (x, y, z) with the unit normals of its cell's two
// triangles (src/module/boundary.hpp:600-645); same layout as the host's.
struct Bdry3PtDev {
    double x[3], n1[3], n2[3];
    double noden[3];                 // node normal (curvilinear 'C' grids)
    double zxx, zxy, zyy;            // depth curvatures of the cell ('C'; 0 otherwise)
    double kxx, kxy, kyy;            // angle curvatures of the cell ('C'; 0 otherwise)
};

// Preprocessed 3-D environment (BELLHOP3D field modes) for one frequency.
struct Env3Dev {
    EnvDev e1d;                      // 1-D SSP tables (ssp_type, nssp, z, rho, c, ...); hexahedral uses z, rho
    int32_t hex, hnx, hny, hnz;      // hexahedral grid (src/ssp.hpp:220-305)
    const double *hx, *hy, *hz, *hc, *hcz;
    HsDev top, bot;
    int32_t top_nx, top_ny, bot_nx, bot_ny;
    int32_t top_curv, bot_curv;      // 'C' grids: normals and curvature interpolated at reflections
    const Bdry3PtDev *btop, *bbot;
    int32_t nsx, nsy, nsz, nrr, nrz, ntheta, nalpha, nbeta, isingle_alpha, isingle_beta;
    const double *sx, *sy, *rr, *tcs;   // tcs: receiver bearing (cos, sin) pairs
    const double *alpha, *beta;
    const double *acs, *bcs;            // (cos, sin) pairs of alpha and beta, from the host's libm
    int32_t nx2d;                       // RunType(6) '2': 2-D rays in the bearing planes
    const float *sz, *rz;
    double dalpha, dbeta, deltas, box_x, box_y, box_z, freq0;
    int32_t gaussian, coherent, run0, nsbp;
    const double *sbp;
};

// One 3-D influence segment (point0 -> point1 of Step_InfluenceGeoCart, 3-D
// branch, src/influence.hpp:1201-1406) after the receiver-range walk.
struct alignas(16) SegRec3 {
    double x0[3];              // point0.x
    double tau0r, tau0i, dtaur, dtaui;
    double rayt[3], e1[3], e2[3];   // unit tangent, ray normals (RayNormal_unit at point1.phi)
    double rlen;
    double q0[4], dq[4];       // point0.q, point1.q - point0.q, m[col][row] as glm
    double rcp_q0, rcp_qhat0;  // Dalpha / c0, |cos alpha| Dbeta / c0 of the ray
    double cnst_num;           // Ratio1 * point1.c * point1.Amp
    double phase0;             // point0.Phase + inflray.phase
    double qold;               // det(point0.q): caustic reference of FinalPhase
    double ldiag;              // L_diag beam radius bound
    double zlo, zhi;           // min / max depth of the segment
    int32_t ir_lo, ir_hi, job, is;
    int32_t ntop, nbot;        // point1's bounce counts (arrivals)
};

struct GroupDev {
    const EnvDev *env;       // device pointer
    int64_t job_base;        // first job index of this group
    int32_t njobs;           // nsz_or_1 * nalpha_or_1
    int32_t nfreq;           // frequencies evaluated from this group's trajectories
    int32_t freq_base;       // index of first frequency slot in the launch's freq list
    int32_t field_stride_f;  // complex elements per frequency field of this group
    int64_t field_base;      // offset (complex elements) of this group's first field
    // influence accumulator layout [field][isz][ir][iz], depth rows acc_nz long
    // (rectilinear grids: nrz rounded up to even, so depth pairs are 16-byte
    // aligned); acc_base is even
    int64_t acc_base;
    int64_t acc_stride_f;    // accumulator elements per frequency field
    int32_t acc_nz;
    int32_t field_index;     // index of the group's first field in the launch
    const Env3Dev *env3;     // 3-D groups: the environment (env is then null)
};

// One influence segment (point0 -> point1 of Step_InfluenceGeoCart,
// src/influence.hpp:1201-1406), with the receiver-column walk already done.
// 16-byte aligned (128 B mixed, 192 B FP64) so that a record is written with
// full 16-byte stores.
template<typename R> struct alignas(16) SegRec {
    double x0r, x0z;      // point0.x
    double tau0r;         // point0.tau.real()
    R dtaur, tau0i, dtaui;
    R tx, tz;             // unit ray tangent (rayt)
    R rlen;               // segment length
    R q0, dq;             // point0.q.x, point1.q.x - point0.q.x
    R rcp_q0;             // Dalpha / c0 of the ray
    R cnst_num;           // Ratio1 * sqrt(point1.c) * point1.Amp
    R phase_a;            // (Gaussian ? point1 : point0).Phase + inflray.phase
    R phase_b;            // inflray.phase + pi/2 (caustic branch of FinalPhase)
    R sigma_seg;          // max|q| * rcp_q0 / |rayt.x| before AdjustSigma
    R c0;                 // point0.c (Gaussian AdjustSigma wavelength)
    R tau1r;              // point1.tau.real() (Gaussian AdjustSigma)
    R zlo, zhi;           // min / max depth of the segment
    R rcvr_decl;          // receiver declination angle (deg)
    int32_t ir_lo, ir_hi; // receiver columns evaluated (inclusive), ir_lo <= ir_hi
    int32_t job;          // global job (ray) index
    int32_t is;           // step index along the ray
    int32_t ntop, nbot;   // bounce counts of point1
};

// One arrival (include/bhc/structs.hpp:376-380; 40 bytes, same field order).
struct ArrivalRec {
    int32_t NTopBnc, NBotBnc;
    float SrcDeclAngle, SrcAzimAngle, RcvrDeclAngle, RcvrAzimAngle, a, Phase;
    float delay_re, delay_im;
};
// One eigenray hit (include/bhc/structs.hpp:353-361).
struct EigenHitRec {
    int32_t is, itheta, ir, iz, isx, isy, isz, ialpha, ibeta;
};
// One beam-receiver contribution of an arrivals / eigen run before ordering:
// amplitude cnst * w, phase, complex delay (FP64, as AddArr compares them),
// receiver angle, bounce counts, global job and launch-angle index. Eigen runs
// reuse ntop / nbot / job for the step, range index and (depth | source << 20).
struct ArrCand {
    double amp, phase, delay_re, delay_im;
    float rcvr_decl;
    int32_t ntop, nbot, job, aux;
    float rcvr_azim;           // 3-D: receiver azimuth (deg); 2-D: unused
};
// Influence types beyond geometric Cartesian (src/influence.hpp:1495-1536):
// geometric hat / Gaussian in ray-centred coordinates ('g', 'b'), Cerveny
// paraxial beams in ray-centred ('R') and Cartesian ('C') coordinates, and
// simple Gaussian beams ('S').
enum InflKind : int32_t { INFL_GEO_CART = 0, INFL_GEO_RAYCEN = 1, INFL_CERV_RAYCEN = 2, INFL_CERV_CART = 3,
                          INFL_SGB = 4 };

// One influence record of those types (FP64). Ray-centred kinds store one
// record per ray segment (point A = the last valid point and its ray normal,
// point B = point1); the receiver ranges between the two normals depend on the
// receiver depth and are found per depth by the influence kernel. Cartesian
// Cerveny and simple Gaussian beams store one record per bracketed receiver
// range (column), with the ray quantities interpolated to it, because their
// receiver walk carries state along the ray.
struct alignas(16) XSeg {
    double xa, za, nxa, nza;       // ray-centred: point A and its ray normal
    double xb, zb, nxb, nzb;       // ray-centred: point B and its normal; columns: x, z at the column
    double tau0r, tau0i, dtaur, dtaui;   // delay at A (columns: at the column), change from A to B
    double q0r, q0i, dqr, dqi;     // geometric q (real) or Cerveny qB at A, change from A to B
    double g0r, g0i, dgr, dgi;     // Cerveny gamma at A (columns: at the column), change from A to B
    double cr, ci;                 // Cartesian Cerveny column: Ratio1 sqrt(c |eps0| / q), KMAH sign
    double amp, ph_a, ph_b;        // geometric: Ratio1 sqrt(c1) Amp1 and the two FinalPhase values;
                                   // Cerveny: (Ratio1) Amp1, Phase1; simple Gaussian: Ratio1 cn Amp1, phase
    double c0, tau1r, rcp_q0, radmax;   // point0.c, point1.tau.real, Dalpha / c0, 50 wavelengths
    double t1x, t1y, eps_abs;      // point1.t (columns: interpolated rayt), Cerveny |eps1|
    double sint, sgb_a, drab, dzab; // simple Gaussian: distance along the ray, beam factor, rB - rA, zB - zA
    double rcvr_decl;              // receiver declination (deg)
    int32_t job, is, ir, ntop, nbot, kmah0, valid, pad;
};

// One 3-D segment of geometric beams in ray-centred coordinates ('g', 'b';
// Step_InfluenceGeoRayCen, 3-D branch, src/influence.hpp:1030-1194): point0
// with the ray normals of the last valid point, point1 with its own normals,
// and what InfluenceGeoCore interpolates between them.
struct alignas(16) XSeg3 {
    double x0[3], n1a[3], n2a[3], ta[3];   // point0.x, inflray.rayn1 / rayn2, point0.c point0.t
    double x1[3], n1b[3], n2b[3], tb[3];   // point1.x, its ray normals, point1.c point1.t
    double q0[4], dq[4];                   // point0.q, point1.q - point0.q (m[col][row] as glm)
    double tau0r, tau0i, dtaur, dtaui;
    double rcp_q0, rcp_qhat0, cnst_num;    // Dalpha / c0, |cos alpha| Dbeta / c0, Ratio1 point1.c point1.Amp
    double phase0, qold;                   // point0.Phase + inflray.phase; det(point0.q) (caustic reference)
    double maxr_m, maxr_n;                 // Gaussian: largest beam radii along the two normals
    double xs, ys;                         // source position
    int32_t job, is, ntop, nbot;
};

// Bit layout of the ordering keys (low to high): arrivals: step | job | cell;
// eigen: depth | walk position | step | job | field (3-D: depth | bearing |
// walk position | step | job | trace group).
struct ArrKeyBits {
    int sh_walk, sh_is, sh_job, sh_cell;
    int total_bits, eigen;
    int sh_theta;              // 3-D eigen: bearing index above the depth bits
};

struct RunCounters {
    unsigned long long nseg;      // segments appended
    unsigned long long nsteps;    // ray steps taken
    unsigned long long nevals;    // beam-receiver contributions applied
    unsigned int err_bits, warn_bits;
    unsigned int overflow_job;    // first job that could not store its segments
    unsigned int pad;
    unsigned long long chunk_counter;   // influence work queue (32-segment chunks)
};

} // namespace bhcb
