// trj_common.cuh -- shared definitions of the sm_100a g(r)/S(Q) library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <string>
#include <unordered_map>

#include "../../include/trj_sm100.h"

// Device-side status word bits (ctx->status_dev[0]); collected by trj_ctx_check.
enum : unsigned {
    TRJ_DEV_BAD_DATA = 1u << 0,      // non-finite coordinate or species out of range
    TRJ_DEV_TIMEOUT = 1u << 1,       // a bounded mbarrier / flag wait ran out
    TRJ_DEV_CAPACITY = 1u << 2,      // more atoms in a cell/tile than staged capacity
    TRJ_DEV_COUNT_MISMATCH = 1u << 3 // species counts differ from the plan's
};

struct trj_ctx {
    int device = 0;
    int sm_count = 0;
    size_t smem_optin = 0;
    unsigned* status_dev = nullptr;     // [0] status bits, [1..7] diagnostics
    unsigned* status_host = nullptr;    // pinned mirror
    struct PackScratch {
        void* ptr = nullptr;
        size_t bytes = 0;
    };
    // per-block species counts of trj_frame_pack, one buffer per stream so that packs on
    // different streams never share scratch
    std::unordered_map<void*, PackScratch> pack_scratch;
    bool timing = false;
    long long launches = 0;             // kernels this library launched on the context
    trj_alloc_fn alloc = nullptr;       // caller-provided device allocator (NULL: cudaMalloc)
    trj_free_fn free_fn = nullptr;
    void* alloc_user = nullptr;
    int sq_tile_cols = 0;               // widest tensor-core S(Q) tile of plans created next (0: 224)
    std::string last_error;
};

// A start/stop CUDA event pair recorded around one kernel launch when timing is on.
struct trj_kernel_timer {
    cudaEvent_t start = nullptr, stop = nullptr;
    bool recorded = false;
    void begin(const trj_ctx* ctx, cudaStream_t s) {
        if (!ctx->timing) return;
        if (!start) {
            cudaEventCreate(&start);
            cudaEventCreate(&stop);
        }
        cudaEventRecord(start, s);
    }
    void end(const trj_ctx* ctx, cudaStream_t s) {
        if (!ctx->timing || !start) return;
        cudaEventRecord(stop, s);
        recorded = true;
    }
    int elapsed(trj_ctx* ctx, float* ms);
    void release() {
        if (start) cudaEventDestroy(start);
        if (stop) cudaEventDestroy(stop);
        start = stop = nullptr;
    }
};

// Device allocation through the context's allocator (cudaMalloc/cudaFree unless one is installed).
inline cudaError_t trj_dev_alloc(trj_ctx* ctx, void** p, size_t bytes) {
    if (ctx->alloc) {
        *p = ctx->alloc(bytes, ctx->alloc_user);
        return *p ? cudaSuccess : cudaErrorMemoryAllocation;
    }
    return cudaMalloc(p, bytes);
}
inline void trj_dev_free(trj_ctx* ctx, void* p) {
    if (!p) return;
    if (ctx->alloc) ctx->free_fn(p, ctx->alloc_user);
    else cudaFree(p);
}

// Records an error message on the context and returns the status code.
int trj_fail(trj_ctx* ctx, int code, const char* fmt, ...);

#define TRJ_CUDA_TRY(ctx, call)                                                        \
    do {                                                                               \
        cudaError_t _e = (call);                                                       \
        if (_e != cudaSuccess)                                                         \
            return trj_fail((ctx), TRJ_ERR_CUDA, "%s failed: %s (%s:%d)", #call,      \
                            cudaGetErrorString(_e), __FILE__, __LINE__);               \
    } while (0)

// Make `device` current for the duration of a call; restores the previous one.
struct trj_device_guard {
    int prev = -1;
    explicit trj_device_guard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~trj_device_guard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// 0-based species pair row: ind_ij of the reference (rdf.cuf:741-753) minus one.
__host__ __device__ __forceinline__ int trj_pair_row(int a, int b, int nsp) {
    if (a > b) { int t = a; a = b; b = t; }
    return a * (nsp - 1) - a * (a - 1) / 2 + b;
}

// FP32 fold of the reference: r - L*int(r/L), each operation rounded once (netcdf.f90:681).
__device__ __forceinline__ float trj_fold_ref(float r, float L) {
    float q = __fdiv_rn(r, L);
    float t = truncf(q);
    return __fsub_rn(r, __fmul_rn(L, t));
}

// Fixed-point phase coordinate of a folded coordinate: frac(x / L) as a 32-bit fraction of a turn,
// rint(frac * 2^32) mod 2^32, in FP64 (so n * u mod 2^32 is the phase of lattice vector n exactly).
__device__ __forceinline__ unsigned trj_phase_fraction(float x, double L) {
    const double s = (double)x / L;
    const double f = s - floor(s);                             // [0, 1]
    return (unsigned)(long long)rint(f * 4294967296.0);        // 2^32 wraps to 0
}

// Bound on any mbarrier wait in this library, in SM clocks (2^32 clocks: about 2 s at 2 GHz).
#define TRJ_WAIT_CLOCKS (1ll << 32)
// Longest single hardware suspension of a waiting thread (ns); it resumes as soon as the phase
// completes, so the value only bounds how often the deadline is checked.
#ifndef TRJ_SUSPEND_NS
#define TRJ_SUSPEND_NS 20000u
#endif

__device__ __forceinline__ void trj_raise(unsigned* status, unsigned bit) {
    atomicOr(status, bit);
}

// ---- mbarrier / bulk-copy helpers (sm_90+ PTX, used on sm_100a) ----------

__device__ __forceinline__ uint32_t trj_smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void trj_mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(trj_smem_addr(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void trj_fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void trj_mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(trj_smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void trj_mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(trj_smem_addr(bar)) : "memory");
}

// Returns true once phase `parity` of the barrier has completed; false after TRJ_WAIT_CLOCKS
// (caller raises TRJ_DEV_TIMEOUT and leaves).  try_wait with a suspend-time hint parks the thread
// in hardware until the phase completes, so a waiting warp issues no polling instructions.
__device__ __forceinline__ bool trj_mbar_wait_limit(uint64_t* bar, unsigned parity, long long limit) {
    const uint32_t addr = trj_smem_addr(bar);
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity), "r"(TRJ_SUSPEND_NS)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > limit) return false;
    }
}

__device__ __forceinline__ bool trj_mbar_wait(uint64_t* bar, unsigned parity) {
    return trj_mbar_wait_limit(bar, parity, TRJ_WAIT_CLOCKS);
}

// 1-D bulk copy global -> shared (TMA engine, no multicast), completion on `bar`.
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void trj_bulk_g2s(void* dst, const void* src, unsigned bytes,
                                             uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            trj_smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(trj_smem_addr(bar))
        : "memory");
}
