/*
 * ORACLE — test infrastructure only. Never linked into or called by the
 * product library; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it, and only as the checker.
 *
 * Plain-C, single-threaded, FP64 restatement of the reference's 2-D BELLHOP
 * beam tracer for the field modes (TL coherent/semi-coherent/incoherent,
 * arrivals, eigenray hits) with geometric hat / Gaussian beams in Cartesian
 * coordinates. Every function cites the reference file:line it follows
 * (paths relative to the reference project root).
 *
 * Parity pin: outputs are checked against the reference's own bellhopcxx,
 * compiled from its unmodified sources by oracle/Makefile, on the same inputs
 * (tests/test_oracle_pin.py and the fixtures in tests/golden/).
 *
 * Inputs are "file-level": the values exactly as the reference's readers
 * produce them from an .env/.bty/.ati/.sbp set (before SubTab, km->m, deg->rad
 * and table building), so this oracle does its own preprocessing.
 */
#ifndef ORACLE2D_H
#define ORACLE2D_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct O2Env {
    /* Run / beam options (module/runtype.hpp, module/beaminfo.hpp) */
    char run_type[7];   /* Beam->RunType as read, e.g. "CG RR  " */
    char ssp_type;      /* TopOpt[0]: N C S P A */
    char top_bc;        /* TopOpt[1]: V R A G */
    char atten_unit[2]; /* TopOpt[2..3] */
    char bot_bc;        /* BotOpt[0] */
    char top_file;      /* TopOpt[4] == '~' or '*' -> altimetry file given */
    char bot_file;      /* BotOpt[1] */
    double freq0;
    /* Francois-Garrison volume attenuation (TopOpt[3] == 'F') */
    double fg_T, fg_S, fg_pH, fg_zbar;
    int32_t nbio;
    const double *bio; /* 5 per layer: z1 z2 f0 q a0 */
    /* halfspaces: zTemp alphaR betaR rho alphaI betaI Mz */
    double top_hs[7], bot_hs[7];
    /* SSP nodes as read (module/ssp.hpp:74-118) */
    int32_t nssp;
    const double *ssp_z, *ssp_alphaR, *ssp_betaR, *ssp_rho, *ssp_alphaI, *ssp_betaI;
    double bot_depth;
    /* boundary files (module/boundary.hpp:85-228): r in km, z in m,
       geo = 5 per point (alphaR betaR rho alphaI betaI) for long format */
    char top_type[2], bot_type[2];
    int32_t ntop, nbot;
    const double *top_r, *top_z, *top_geo;
    const double *bot_r, *bot_z, *bot_geo;
    /* source beam pattern (module/sbp.hpp); nsbp == 0 -> omnidirectional */
    int32_t nsbp;
    const double *sbp; /* pairs: angle(deg), level(dB) */
    /* vectors as read, before SubTab: arrays hold max(3,n) entries with the
       unread slots set to -999.9 as ReadVector does (common_setup.hpp:370-381) */
    int32_t nsz, nrz, nrr, nalpha;
    const float *sz_in, *rz_in;
    const double *rr_in;    /* km */
    const double *alpha_in; /* deg; nalpha == 0 -> EstimateNumAngles */
    int32_t isingle;        /* TopOpt[5] == 'I' single-beam index (1-based), else 0 */
    double deltas, box_z, box_r_km;
    /* arrivals / eigen storage */
    int32_t max_narr, allow_merging, eigen_memsize;
} O2Env;

typedef struct O2Arrival { /* include/bhc/structs.hpp:376-380 */
    int32_t NTopBnc, NBotBnc;
    float SrcDeclAngle, SrcAzimAngle, RcvrDeclAngle, RcvrAzimAngle, a, Phase;
    float delay_re, delay_im;
} O2Arrival;

typedef struct O2Hit { /* include/bhc/structs.hpp:353-361 */
    int32_t is, itheta, ir, iz, isx, isy, isz, ialpha, ibeta;
} O2Hit;

typedef struct O2Out {
    /* sizes (filled by oracle2d_sizes) */
    int32_t NSz, NRz, NRz_per_range, NRr, Nalpha;
    /* caller-allocated outputs (may be NULL when not needed) */
    float *field;      /* [NSz][NRz_per_range][NRr] interleaved re,im */
    int32_t *narr;     /* [NSz][NRz_per_range][NRr] */
    O2Arrival *arr;    /* [NSz][NRz_per_range][NRr][max_narr] */
    O2Hit *hits;       /* [eigen_memsize] */
    int32_t neigen;
    double *rr_m;      /* [NRr] receiver ranges in m, as used */
    float *rz_m;       /* [NRz] receiver depths in m, as used */
    double *alpha_rad; /* [Nalpha] */
    /* counters for throughput accounting */
    int64_t nsteps;    /* ray steps (Step() calls) */
    int64_t nevals;    /* beam-receiver contributions applied */
    uint32_t err_bits, warn_bits;
    int32_t ray_first, ray_count; /* optional sub-range of rays (count<=0 -> all) */
} O2Out;

/* Fill the size fields of out from env (runs the vector preprocessing). */
int oracle2d_sizes(const O2Env *env, O2Out *out);
/* Run the trace + influence + postprocess. Returns 0 on success. */
int oracle2d_run(const O2Env *env, O2Out *out);

#ifdef __cplusplus
}
#endif
#endif
