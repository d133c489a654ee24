// Shared-memory staging of the tables the 2-D ray step reads (SSP nodes and
// coefficients, boundary nodes, receiver ranges) with the Tensor Memory
// Accelerator's bulk copies (cp.async.bulk, completion counted on an
// mbarrier in bytes).
//
// Each trace CTA stages the environment of the ray group it starts in: one
// thread issues one bulk copy per table that fits the shared-memory budget,
// in the order below, and the CTA waits for the transaction count with a
// bounded wait. Rays of that group then read the tables from shared memory
// through a copy of the environment whose table pointers are rewritten to the
// shared copies; rays of other groups, and tables that do not fit, read
// global memory as before. A bulk copy needs 16-byte aligned addresses and a
// multiple of 16 bytes: the host arena places every table at a 256-byte
// offset and pads its size to 16 bytes.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include "bhcb_internal.h"

namespace bhcb {

// in the order of their reads per step: SSP nodes and coefficients (three
// evaluations per step), boundary nodes (segment checks), receiver ranges
enum StageTable : int { ST_Z, ST_C, ST_CZ, ST_COEF, ST_N2, ST_N2Z, ST_RHO, ST_QR, ST_QC, ST_QCZ, ST_BTOP, ST_BBOT,
                        ST_RR, ST_COUNT };

__host__ __device__ inline size_t round16(size_t b) { return (b + 15) & ~size_t(15); }

// most shared memory a trace CTA stages, and the default
constexpr unsigned int STAGE_MAX_BYTES = 64u * 1024u;
constexpr unsigned int STAGE_DEFAULT_BYTES = 32u * 1024u;

// bytes of each table the step of this environment's SSP type reads (0: not read)
__host__ __device__ inline void stage_table_bytes(const EnvDev &e, size_t b[ST_COUNT])
{
    for(int k = 0; k < ST_COUNT; ++k) b[k] = 0;
    const size_t n = (size_t)e.nssp;
    const int t = e.ssp_type;
    if(t != SSP_ANALYTIC) {
        b[ST_Z] = n * 8;
        b[ST_RHO] = n * 8;   // reflections (and N2-linear) interpolate the density
    }
    if(t == SSP_CLINEAR || t == SSP_QUAD) {
        b[ST_C] = 2 * n * 8;
        if(t == SSP_CLINEAR) b[ST_CZ] = 2 * n * 8;
    }
    if(t == SSP_CUBIC || t == SSP_PCHIP) b[ST_COEF] = 8 * n * 8;
    if(t == SSP_N2LINEAR) {
        b[ST_N2] = 2 * n * 8;
        b[ST_N2Z] = 2 * n * 8;
    }
    if(t == SSP_QUAD) {
        b[ST_QR] = (size_t)e.nqr * 8;
        b[ST_QC] = n * (size_t)e.nqr * 8;
        b[ST_QCZ] = n * (size_t)e.nqr * 8;
    }
    b[ST_BBOT] = (size_t)e.nbot * sizeof(BdryPtDev);
    b[ST_BTOP] = (size_t)e.ntop * sizeof(BdryPtDev);
    b[ST_RR] = (size_t)e.nrr * 8;
}

// shared-memory offsets of the tables that fit in budget (SIZE_MAX: stays in
// global memory); returns the bytes used
__host__ __device__ inline size_t stage_plan(const EnvDev &e, size_t budget, size_t off[ST_COUNT])
{
    size_t b[ST_COUNT];
    stage_table_bytes(e, b);
    size_t used = 0;
    for(int k = 0; k < ST_COUNT; ++k) {
        off[k] = (size_t)-1;
        const size_t r = round16(b[k]);
        if(r == 0 || used + r > budget) continue;
        off[k] = used;
        used += r;
    }
    return used;
}

#ifdef __CUDACC__
namespace stage_detail {
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.b32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_addr(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}
// bulk copy global -> this CTA's shared memory, completion on bar
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
} // namespace stage_detail

// Limit of the staging wait (try_wait polls); a copy of a few tens of KB
// completes in microseconds, so running out means something is wrong.
constexpr unsigned STAGE_WAIT_LIMIT = 1u << 22;

// Called by every thread of the CTA. Thread 0 copies *src into s_env, plans
// the tables, rewrites s_env's pointers to the staged copies and issues the
// bulk copies; all threads then wait for them. Returns false (and sets
// ERR_STAGE_WAIT) when the wait ran out: the caller then reads global memory.
__device__ __forceinline__ bool stage_env_tables(const EnvDev *src, EnvDev &s_env, unsigned char *s_tab,
                                                 size_t budget, uint64_t *s_bar, RunCounters *ctr)
{
    using namespace stage_detail;
    if(threadIdx.x == 0) {
        s_env = *src;
        size_t off[ST_COUNT], b[ST_COUNT];
        const size_t total = stage_plan(s_env, budget, off);
        stage_table_bytes(s_env, b);
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(s_bar)), "r"(1u) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(s_bar)),
                     "r"((uint32_t)total)
                     : "memory");
        const void *srcs[ST_COUNT] = {s_env.z, s_env.c, s_env.cz, s_env.coef, s_env.n2, s_env.n2z, s_env.rho,
                                      s_env.qr, s_env.qc, s_env.qcz, s_env.btop, s_env.bbot, s_env.rr};
        for(int k = 0; k < ST_COUNT; ++k) {
            if(off[k] == (size_t)-1) continue;
            bulk_g2s(s_tab + off[k], srcs[k], (uint32_t)round16(b[k]), s_bar);
        }
        auto at = [&](int k) -> const void * { return off[k] == (size_t)-1 ? nullptr : s_tab + off[k]; };
        if(at(ST_Z)) s_env.z = (const double *)at(ST_Z);
        if(at(ST_C)) s_env.c = (const double *)at(ST_C);
        if(at(ST_CZ)) s_env.cz = (const double *)at(ST_CZ);
        if(at(ST_COEF)) s_env.coef = (const double *)at(ST_COEF);
        if(at(ST_N2)) s_env.n2 = (const double *)at(ST_N2);
        if(at(ST_N2Z)) s_env.n2z = (const double *)at(ST_N2Z);
        if(at(ST_RHO)) s_env.rho = (const double *)at(ST_RHO);
        if(at(ST_QR)) s_env.qr = (const double *)at(ST_QR);
        if(at(ST_QC)) s_env.qc = (const double *)at(ST_QC);
        if(at(ST_QCZ)) s_env.qcz = (const double *)at(ST_QCZ);
        if(at(ST_BBOT)) s_env.bbot = (const BdryPtDev *)at(ST_BBOT);
        if(at(ST_BTOP)) s_env.btop = (const BdryPtDev *)at(ST_BTOP);
        if(at(ST_RR)) s_env.rr = (const double *)at(ST_RR);
    }
    __syncthreads();
    bool ok = false;
    for(unsigned i = 0; i < STAGE_WAIT_LIMIT; ++i)
        if(mbar_try_wait(s_bar, 0)) { ok = true; break; }
    if(!ok && threadIdx.x == 0) atomicOr(&ctr->err_bits, 1u << ERR_STAGE_WAIT);
    return ok;
}

// Before the CTA exits: once more, bounded, for copies still in flight after
// a wait that ran out.
__device__ __forceinline__ void stage_drain(uint64_t *s_bar)
{
    for(unsigned i = 0; i < STAGE_WAIT_LIMIT; ++i)
        if(stage_detail::mbar_try_wait(s_bar, 0)) return;
}
#endif

} // namespace bhcb
