/*
 * bhcb — C ABI of the B200 beam tracer (libbhcb.so).
 *
 * The reference exposes its tracer as C++ templates in include/bhc/bhc.hpp
 * (bhc::setup / run / writeout / finalize over bhcParams / bhcOutputs). Its
 * internal seam for the field modes is RunFieldModesImpl
 * (src/mode/fieldimpl.hpp:27-28). This header is the plain-C surface that a
 * host binding (C++, ctypes, cgo, JNI) calls instead; each entry point names
 * the reference call it replaces.
 *
 * Conventions: every function returns 0 on success and a non-zero status on
 * failure (never throws, never resets the device); the message is available
 * from bhcb_last_error. A context is bound to one GPU and one CUDA stream and
 * is not thread-safe; separate contexts are independent (the reference's
 * "multiple instances" rule, include/bhc/bhc.hpp:41-43).
 */
#ifndef BHCB_H
#define BHCB_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bhcb_ctx bhcb_ctx;

enum {
    BHCB_OK = 0,
    BHCB_ERR_ARG = 1,        /* invalid argument */
    BHCB_ERR_INPUT = 2,      /* invalid or unsupported environment */
    BHCB_ERR_CUDA = 3,       /* CUDA runtime error (context stays usable) */
    BHCB_ERR_RUN = 4,        /* tracer reported an error bit (see err_bits) */
    BHCB_ERR_MEMORY = 5,     /* max_memory budget exceeded */
    BHCB_ERR_STATE = 6       /* call out of order (e.g. run before setup) */
};

enum { BHCB_PREC_FP64 = 0, BHCB_PREC_MIXED = 1 };

/* TL runs evaluate the influence after the trace in stream order (the
   default; this flag is kept for callers that set it). bhcb_launch then only
   enqueues work: its first launch after bhcb_prepare runs the kernels
   directly, the second captures the step (counter set-up, trace, influence,
   ScalePressure) into a CUDA graph, and later launches replay that graph. */
#define BHCB_FLAG_SERIAL_INFLUENCE 1
/* Mixed-precision TL runs overlap the influence with the trace: bhcb_run and
   bhcb_launch relaunch influence kernels on a second stream for the segment
   blocks the running trace has published, so bhcb_launch returns only once the
   trace has ended (the final influence and scale kernels are still enqueued,
   not waited for). Not captured in a graph. On B200 the concurrent influence
   slows the latency-bound trace, so this is off unless asked for. */
#define BHCB_FLAG_OVERLAP_INFLUENCE 2
/* Launch the kernels of every step directly instead of replaying a CUDA graph. */
#define BHCB_FLAG_NO_GRAPH 4
/* Pipelined TL steps (geometric Cartesian beams): successive bhcb_launch
   calls of a prepared batch go in pairs whose two traces run at the same time
   (internal streams, one buffer slot of segment records, counters and
   accumulator each: twice their device memory), then their influence and
   ScalePressure one after the other; the next pair's traces start when the
   pair's last scale ends. bhcb_launch returns at once; work enqueued on the
   context stream after a launch waits for that launch's fields; bhcb_sync
   waits for every launch. The first launch after bhcb_prepare or bhcb_sync is
   ordered after the work already on the context stream; later launches are
   not, until the next bhcb_sync. */
#define BHCB_FLAG_PIPELINE 8

/* Context options; mirrors bhcInit (include/bhc/structs.hpp:490-546). */
typedef struct bhcb_init {
    int32_t gpu_index;        /* bhcInit::gpuIndex */
    int32_t precision;        /* BHCB_PREC_FP64 or BHCB_PREC_MIXED */
    uint64_t max_memory;      /* bhcInit::maxMemory (device bytes); 0 = 16 GiB */
    int32_t share_trajectory; /* frequencies share one trace when tables allow (mixed only) */
    int32_t flags;            /* BHCB_FLAG_* */
    void (*output_callback)(const char *message); /* bhcInit::outputCallback */
} bhcb_init;

/* Counters of the last run. */
typedef struct bhcb_stats {
    uint64_t rays, steps, segments, evals;
    uint32_t err_bits, warn_bits;   /* reference ErrState bit numbering (src/util/errors.hpp:61-93) */
    int32_t groups, fields;         /* trace groups launched, TL fields produced */
    double trace_ms, influence_ms, total_ms;   /* influence_ms: influence time after the trace ended */
    uint64_t h2d_bytes;             /* table bytes uploaded by the last bhcb_prepare */
    double influence_span_ms;       /* first influence launch to the last one's end (overlapped runs) */
} bhcb_stats;

/* Create a context; replaces the bhcInternal construction in bhc::setup
   (src/api.cpp:194-215, setupGPU src/api.cpp:144-189). init may be NULL. */
int bhcb_open(const bhcb_init *init, bhcb_ctx **out);

/* bhc::finalize (src/api.cpp:830-855): release every resource. */
void bhcb_close(bhcb_ctx *ctx);

/* bhc::setup with bhcInit::FileRoot set (src/api.cpp:194-291): read
   FileRoot.env (+ .bty/.ati/.sbp) as the context's single environment. */
int bhcb_setup(bhcb_ctx *ctx, const char *file_root);

/* Batched extension (no reference counterpart: the reference needs one
   bhcParams per environment): append one more environment; returns its index
   in *env_index. bhcb_setup is bhcb_clear + bhcb_add_env. */
int bhcb_add_env(bhcb_ctx *ctx, const char *file_root, int32_t *env_index);
int bhcb_clear(bhcb_ctx *ctx);

/* In-memory 2-D environment (the values bhcParams<false> holds after
   bhc::setup and the extsetup_* calls, include/bhc/bhc.hpp:58-452; the .env
   grammar's values, src/api.cpp:253-277). Vectors are complete (not
   sub-tabulated): nsz source depths (m), nrz receiver depths (m), nrr ranges
   (km), nalpha launch angles (degrees; nalpha 0 = estimated as
   EstimateNumAngles does, src/module/rayangles.hpp:212-238, over -20..20). An
   altimetry / bathymetry with 0 points is flat. All arrays are read during
   the call only. */
typedef struct bhcb_env_desc {
    const char *title;
    double freq0;
    char top_opt[6], bot_opt[6];        /* TopOpt, BotOpt (SSP type, bc, atten units, ...) */
    double fg[4];                       /* Francois-Garrison T, S, pH, z_bar (TopOpt[3] 'F') */
    int32_t nbio;                       /* biological layers (TopOpt[3] 'B'): 5 doubles each */
    const double *bio;                  /* z1 z2 f0 q a0 */
    double top_hs[7], bot_hs[7];        /* halfspaces: zTemp alphaR betaR rho alphaI betaI Mz */
    int32_t nssp;                       /* SSP nodes */
    const double *ssp_z, *ssp_alphaR, *ssp_betaR, *ssp_rho, *ssp_alphaI, *ssp_betaI;
    double bot_depth;                   /* depth of the bottom (m) */
    char ati_type[2], bty_type[2];      /* boundary file types ('L' / 'C', 'S' / 'L') */
    int32_t nati, nbty;                 /* points; 0 = flat boundary */
    const double *ati_r_km, *ati_z, *ati_geo;   /* geo: 5 per point (long format), may be NULL */
    const double *bty_r_km, *bty_z, *bty_geo;
    int32_t nsbp;                       /* source beam pattern points (0 = omnidirectional) */
    const double *sbp;                  /* (angle deg, level dB) pairs */
    int32_t nsz, nrz, nrr, nalpha, isingle;
    const float *sz, *rz;
    const double *rr_km, *alpha_deg;
    char run_type[7];                   /* Beam->RunType */
    char cerv_type[2];                  /* Cerveny beam width / curvature options (Beam->Type[1..2]) */
    double deltas, box_z, box_r_km;     /* step (m, 0 = automatic), beam box */
    double eps_mult, rloop;             /* Cerveny epsilon multiplier and rLoop */
    int32_t nimage, ibeam_window;
    char component;
    int32_t nquad_r;                    /* quad SSP ('Q'): ranges (km) and c[iz * nquad_r + ir] */
    const double *quad_r_km, *quad_c;
    int32_t nbrc, ntrc;                 /* reflection tables ('F'): (theta deg, |R|, phase deg) triples */
    const double *brc, *trc;
} bhcb_env_desc;
/* bhc::setup from parameters in memory (the extsetup_* route): append the
   environment described by desc, like bhcb_add_env does for a file. */
int bhcb_add_env_desc(bhcb_ctx *ctx, const bhcb_env_desc *desc, int32_t *env_index);
/* Read FileRoot.env (+ side files) as a 2-D environment into a descriptor the
   library allocates (arrays included); release it with bhcb_free_env_desc.
   Needs no GPU. msg (may be NULL) receives the reason of a failure. */
int bhcb_read_env_desc(const char *file_root, bhcb_env_desc **desc, char *msg, size_t n);
void bhcb_free_env_desc(bhcb_env_desc *desc);
/* bhc::get_ssp (include/bhc/bhc.hpp:440-452): sound speed (m/s) of
   environment env_index at range r (m) and depth z (m), interpolated as the
   tracer does (SSP types N, C, S, P, Q). Needs no GPU. */
int bhcb_ssp_at(bhcb_ctx *ctx, int32_t env_index, double r, double z, double *c);

/* Multi-frequency extension (no reference counterpart: the reference traces
   one freq0 per bhc::run, include/bhc/bhc.hpp:174-179): evaluate env_index at
   the nfreq given frequencies instead of its file frequency. */
int bhcb_set_frequencies(bhcb_ctx *ctx, int32_t env_index, int32_t nfreq, const double *freqs);

/* bhc::run (src/api.cpp:384-418): preprocess, trace, accumulate and
   post-process (ScalePressure) every field, synchronously. */
int bhcb_run(bhcb_ctx *ctx);

/* Split form of bhcb_run for callers that manage timing / streams:
   bhcb_prepare uploads the tables and sizes the buffers; bhcb_launch enqueues
   the kernels on the context stream without synchronising; bhcb_sync waits
   and checks the run's error bits. */
int bhcb_prepare(bhcb_ctx *ctx);
int bhcb_launch(bhcb_ctx *ctx);
int bhcb_sync(bhcb_ctx *ctx);

/* Output description: outputs.uAllSources layout per field is
   [NSz][NRz_per_range][NRr] complex float (GetFieldAddr, src/common.hpp:393-405). */
int bhcb_field_shape(bhcb_ctx *ctx, int32_t env_index, int32_t *nfreq, int32_t *nsz,
                     int32_t *nrz_per_range, int32_t *nrr);
/* Copy field (env_index, ifreq) to host memory dst (bytes >= its size). */
int bhcb_copy_field(bhcb_ctx *ctx, int32_t env_index, int32_t ifreq, void *dst, size_t bytes);
/* Device pointer of field (env_index, ifreq); valid until the next run/close. */
int bhcb_field_device(bhcb_ctx *ctx, int32_t env_index, int32_t ifreq, void **dptr);
/* Receiver grid as used by the run (ranges in m, depths in m). */
int bhcb_receivers(bhcb_ctx *ctx, int32_t env_index, double *rr, int32_t nrr, float *rz,
                   int32_t nrz);

/* bhc::writeout (src/api.cpp:465-486): TL runs write FileRoot.shd of
   (env_index, ifreq) in the reference's .shd layout (src/mode/tl.cpp:38-248);
   arrivals runs write FileRoot.arr (WriteOutArrivals, src/mode/arr.cpp:88-239:
   Fortran unformatted records for 'a', list-directed text for 'A'). */
int bhcb_writeout(bhcb_ctx *ctx, int32_t env_index, int32_t ifreq, const char *file_root);

/* Arrivals (RunType 'A' / 'a') and eigenray hits ('E'). Arrivals follow
   AddArr (src/arrivals.hpp:45-132) in the reference's single-threaded order
   (ray by ray in job order, step by step), so merging (allow_merging, the
   reference's AllowMerging, src/mode/arr.hpp:78) is deterministic. */
typedef struct bhcb_arrival {   /* Arrival, include/bhc/structs.hpp:376-380 */
    int32_t ntop, nbot;
    float src_decl, src_azim, rcvr_decl, rcvr_azim, a, phase;   /* degrees; phase in radians */
    float delay_re, delay_im;                                   /* complex delay (s) */
} bhcb_arrival;
typedef struct bhcb_eigen_hit { /* EigenHit, include/bhc/structs.hpp:353-361 */
    int32_t is, itheta, ir, iz, isx, isy, isz, ialpha, ibeta;
} bhcb_eigen_hit;
/* Arrival storage per receiver (ArrInfo::MaxNArr; 0 = sized from max_memory like
   src/mode/arr.hpp:80-98, at most 1000) and merging; takes effect at the next prepare. */
int bhcb_set_arrival_options(bhcb_ctx *ctx, int32_t max_narr, int32_t allow_merging);
/* outputs.arrinfo layout per field: NArr [NSz][NRz_per_range][NRr] int32 and
   Arr [same][max_narr] bhcb_arrival, amplitudes scaled (PostProcessArrivals,
   src/mode/arr.cpp:24-74). */
int bhcb_arrivals_shape(bhcb_ctx *ctx, int32_t env_index, int32_t ifreq, int32_t *nsz,
                        int32_t *nrz_per_range, int32_t *nrr, int32_t *max_narr);
int bhcb_copy_arrivals(bhcb_ctx *ctx, int32_t env_index, int32_t ifreq, int32_t *narr, size_t narr_bytes,
                       bhcb_arrival *arr, size_t arr_bytes);
/* outputs.eigen->hits of (env_index, ifreq) in the reference's single-threaded
   order; *nhits = their number, at most max_hits are copied. */
int bhcb_eigen_hits(bhcb_ctx *ctx, int32_t env_index, int32_t ifreq, bhcb_eigen_hit *hits,
                    int64_t max_hits, int64_t *nhits);

/* The context's CUDA stream (cudaStream_t), for callers that time or order
   their own work against the tracer's kernels. */
int bhcb_stream(bhcb_ctx *ctx, void **stream);

/* Counters of the last run. */
int bhcb_get_stats(bhcb_ctx *ctx, bhcb_stats *stats);

/* Last error message (NUL-terminated, truncated to n) and ErrState bits. */
int bhcb_last_error(bhcb_ctx *ctx, char *msg, size_t n, uint32_t *err_bits,
                    uint32_t *warn_bits);

/* Host-only validation (no GPU needed): read FileRoot.env (+ side files) and
   run the preprocessing that bhc::setup's Validate/Echo pass performs
   (src/api.cpp:278-281); report the sizes the run would use. */
typedef struct bhcb_env_info {
    int32_t nsz, nrz, nrz_per_range, nrr, nalpha, ssp_type;
    double freq, deltas;
    char run_type[8], beam_type[8];
} bhcb_env_info;
int bhcb_check_env(const char *file_root, bhcb_env_info *info, char *msg, size_t n);
/* The same check for a 3-D environment: dims as bhcb_field_shape3d, nrays
   the number of rays (jobs) the run traces. Needs no GPU. */
int bhcb_check_env3d(const char *file_root, int32_t *dims, int64_t *nrays, char *msg, size_t n);

/* Allocation-free run (no counterpart in the reference). For callers that
   must not allocate device memory once running — work inside a budget owned
   by another allocator, allocation-free real-time loops. Computes TL field
   (env_index, ifreq) of a context prepared earlier for a TL run (bhcb_prepare
   / bhcb_run, which allocate; other run types give BHCB_ERR_STATE) into the
   caller's device buffer field_dev ([NSz][NRz_per_range][NRr] complex float,
   bytes >= its size, on the context's GPU) on the context stream, then
   synchronises; it is not meant for stream capture (bhcb_graph_* is). It
   runs on the context's GPU whatever device is current and restores the
   current device. It calls no cudaMalloc / cudaFree: its scratch
   (accumulator, counters, field descriptor) is a static device array the
   library reserves on every GPU that loads it, limited to
   BHCB_NOALLOC_MAX_FIELD receivers per field; larger fields are rejected with
   BHCB_ERR_ARG. The first call on a device looks up the array's address
   (cudaGetSymbolAddress). All calls on a device share the array: calls whose
   GPU work overlaps race and must be serialised. msg (may be NULL) receives
   the reason of a failure. */
#define BHCB_NOALLOC_MAX_FIELD (1 << 21)
int bhcb_run_noalloc(bhcb_ctx *ctx, int32_t env_index, int32_t ifreq, void *field_dev, size_t bytes,
                     char *msg, size_t msg_len);

/* BELLHOP3D field modes (bhc::setup / run / writeout with O3D = R3D = true).
   A context holds either 2-D or 3-D environments (bhcb_clear switches).
   Supported: RunType 'C' / 'S' / 'I' with RunType(6) = '3', Cartesian
   geometric hat ('G', '^', ' ') and Gaussian ('B') beams, 1-D profiles
   ('C', 'N', 'S', 'P') or the hexahedral grid ('H', src/ssp.hpp:215-305),
   flat or 'R' gridded altimetry / bathymetry (src/boundary.hpp:66-160),
   boundary conditions 'V', 'R', 'A', 'G'. bhcb_run / bhcb_launch trace and
   evaluate the whole batch; bhcb_copy_field, bhcb_field_device and
   bhcb_writeout take ifreq 0. */
/* bhc::setup<true, true> (src/api.cpp:217-298) on FileRoot.env as a 3-D run. */
int bhcb_setup3d(bhcb_ctx *ctx, const char *file_root);
/* Append another 3-D environment to the batch. */
int bhcb_add_env3d(bhcb_ctx *ctx, const char *file_root, int32_t *env_index);
/* Field layout [NSz][NSx][NSy][Ntheta][NRz][NRr] complex float (GetFieldAddr,
   src/common.hpp:393-405); dims = {NSz, NSx, NSy, Ntheta, NRz, NRr}. */
int bhcb_field_shape3d(bhcb_ctx *ctx, int32_t env_index, int32_t *dims);
/* Source and receiver coordinates of a 3-D environment (Position,
   include/bhc/structs.hpp:278-295): Sx, Sy, Rr in m, Sz, Rz in m, theta in
   degrees; each pointer may be NULL, sizes from bhcb_field_shape3d. */
int bhcb_grid3d(bhcb_ctx *ctx, int32_t env_index, double *sx, double *sy, float *sz, double *rr, float *rz,
                double *theta);

/* CUDA graphs of the hot path (no reference counterpart): one field of a
   prepared context (bhcb_prepare done, TL run) captured into a graph that
   writes into field_dev. The graph owns its scratch (allocated here, before
   the capture); each launch re-clears it, so a graph can be replayed any
   number of times, and graphs of different fields concurrently. Launch on
   `stream` (a cudaStream_t; NULL = the graph's own stream). bhcb_graph_status
   waits for that stream and reports the tracer's error bits and the number
   of contributions of the last launch. */
typedef struct bhcb_graph bhcb_graph;
int bhcb_graph_create(bhcb_ctx *ctx, int32_t env_index, int32_t ifreq, void *field_dev, size_t bytes,
                      bhcb_graph **graph, char *msg, size_t msg_len);
int bhcb_graph_launch(bhcb_graph *graph, void *stream);
int bhcb_graph_status(bhcb_graph *graph, void *stream, uint32_t *err_bits, uint64_t *evals);
void bhcb_graph_destroy(bhcb_graph *graph);

/* Tensor-core GEMM of the TL surrogate (no reference counterpart):
   C[M,N] = epi(A[M,K] * B[N,K]^T), A and B row-major bf16 with K a multiple of
   8 and 16-byte aligned bases, FP32 accumulation in tensor memory (tcgen05).
   Epilogues: F32 (C float, + bias[N] if bias), BF16 (C bf16, + bias), BF16_GELU
   (pre = acc + bias stored to aux_out if not NULL, C = gelu(pre), tanh form),
   BF16_DGELU (C = acc * gelu'(aux_in), aux_in bf16 [M,N]). Enqueued on
   `stream` (a cudaStream_t, NULL = legacy default). bhcb_nn_status reports
   (and optionally clears) the sticky error word a kernel sets when one of its
   bounded waits ran out. */
enum { BHCB_NN_EPI_F32 = 0, BHCB_NN_EPI_BF16 = 1, BHCB_NN_EPI_BF16_GELU = 2, BHCB_NN_EPI_BF16_DGELU = 3 };
int bhcb_nn_gemm(const void *A, const void *B, void *C, int32_t M, int32_t N, int32_t K, int32_t epi,
                 const float *bias, const void *aux_in, void *aux_out, void *stream);
int bhcb_nn_status(int32_t *error, int32_t clear);
/* Surrogate training / inference helpers (device pointers, enqueued on stream):
   tl_db: TL = -20 log10|p| of n complex64 pressures, clamped to [lo, hi];
   transpose: bf16 [rows][cols] -> [cols][rows];
   mse: grad = bf16(scale * 2 (pred - target)), *loss_dev += sum (pred - target)^2;
   row_rms: per-row RMS of pred - target (rows x cols float);
   colsum: db[n] = sum_m dy[m][n] (bf16 in, float out);
   adam: bias-corrected Adam step `step` (1-based) with decoupled weight decay on
   FP32 master weights [rows][cols], refreshing the bf16 copy w_bf16 and, if
   not NULL, its transpose wt_bf16 [cols][rows];
   to_bf16: float -> bf16. */
int bhcb_nn_tl_db(const void *field, float *tl, int64_t n, float lo, float hi, void *stream);
int bhcb_nn_transpose(const void *in, void *out, int32_t rows, int32_t cols, void *stream);
int bhcb_nn_mse(const float *pred, const float *target, int64_t n, float scale, void *grad, double *loss_dev,
                void *stream);
int bhcb_nn_row_rms(const float *pred, const float *target, int32_t rows, int32_t cols, float *rms, void *stream);
int bhcb_nn_colsum(const void *dy, int32_t M, int32_t N, float *db, void *stream);
int bhcb_nn_adam(float *w, const float *g, float *m, float *v, int32_t rows, int32_t cols, float lr, float beta1,
                 float beta2, float eps, int32_t step, float weight_decay, void *w_bf16, void *wt_bf16, void *stream);
int bhcb_nn_to_bf16(const float *x, void *y, int64_t n, void *stream);
/* x = a * x + b over n floats */
int bhcb_nn_affine(float *x, int64_t n, float a, float b, void *stream);

/* Ray trajectories (2-D and 3-D): RunType 'R' traces every ray (RunRayMode,
   src/mode/ray.cpp:163-198); for eigen runs ('E') the rays of the hits of
   (env_index, ifreq) are re-traced up to their hit (PostProcessEigenrays,
   src/mode/eigen.cpp:63-92) on the first call. bhcb_writeout writes them as
   FileRoot.ray (OpenRAYFile / WriteRay, src/mode/ray.hpp:176-247).
   bhcb_copy_rays: npts[nrays] points per ray, bounces[2 nrays] top / bottom
   bounce counts of the last point, alpha_deg[nrays] take-off declinations
   (degrees), rz the points ray after ray, npoints in total: (r, z) in m,
   2 doubles each, for 2-D contexts; (x, y, z) in m, 3 doubles each, for 3-D
   contexts (ifreq 0). */
int bhcb_rays_shape(bhcb_ctx *ctx, int32_t env_index, int32_t ifreq, int64_t *nrays, int64_t *npoints);
int bhcb_copy_rays(bhcb_ctx *ctx, int32_t env_index, int32_t ifreq, int32_t *npts, int32_t *bounces,
                   double *alpha_deg, double *rz, size_t rz_bytes);

/* Autotuner (no reference counterpart): times the prepared 2-D TL workload
   with each candidate launch shape — trace CTAs of 32 or 64 threads (one ray
   per thread), 0, 32 or 64 KB of environment tables staged in each trace
   CTA's shared memory, 2..12 persistent influence CTAs per SM — `repeats` runs each
   (best of), keeps the fastest shape in the context and reports it. The
   trace and the influence are timed apart (serial influence) during tuning.
   bhcb_set_tuning applies a known shape (e.g. one saved from an earlier
   process) without timing. The runs leave the context's outputs valid. */
typedef struct bhcb_tuning {
    int32_t trace_block;            /* threads per trace CTA */
    int32_t influence_ctas_per_sm;  /* persistent influence CTAs per SM */
    int32_t stage_kb;               /* shared memory (KB, 0..64) a trace CTA stages environment tables into */
    double trace_ms, influence_ms;  /* best times measured with the chosen shape */
    int32_t trace_lanes;            /* rays per trace warp (16 or 32; 0 = 32): fewer rays diverge less per step */
} bhcb_tuning;
int bhcb_autotune(bhcb_ctx *ctx, int32_t repeats, bhcb_tuning *out);
int bhcb_set_tuning(bhcb_ctx *ctx, const bhcb_tuning *tuning);

/* Library version string. */
const char *bhcb_version(void);

#ifdef __cplusplus
}
#endif
#endif
