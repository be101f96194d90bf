// sq_tc.cu -- tensor-core S(Q): rho_a(k) for a compact k-region as a BF16 tcgen05 contraction.
//
// For lattice vectors k = 2 pi (nx/Lx, ny/Ly, nz/Lz) the phase factor separates:
//   e^{i k.r_j} = X_j[nx] * Y_j[ny] * Z_j[nz],   X_j[n] = e^{2 pi i n x_j/Lx}, ...
// so for a tile of 128 (nx, ny) rows (16 nx x 8 ny) and a run of nz values,
//   rho(nx, ny, nz) = sum_j A[(nx,ny), j] * Z_j[nz],   A = X*Y,
// a complex GEMM with the atoms as the contraction dimension.  It runs as a real GEMM:
//   K index 2j = Re, 2j+1 = Im of atom j;  B columns 2t (Re out) = (zr, -zi), 2t+1 (Im out) = (zi, zr).
// Each phase value v is split v = hi + lo with hi = bf16(v), lo = bf16(v - hi); the product
// keeps hi*hi + hi*lo + lo*hi (three tcgen05.mma kind::f16 per K-step into one FP32 TMEM
// accumulator).  Every F stages the accumulator is drained and added into an FP64 per-CTA
// block, and the blocks of one species are summed in FP64 in a fixed order.
//
// Phases: every coordinate is the 32-bit fixed-point fraction u = (x/L mod 1) 2^32 (from
// FP64); n*u mod 2^32 in integer arithmetic is exact, and sincospif of the reduced fraction
// gives each factor at FP32 accuracy.
//
// Roles per CTA (320 threads): warps 0-7 generate the A tile (X*Y products, split) in the
// 128-byte-swizzled K-major layout and later drain TMEM; warp 8 streams the B tile (Z phases,
// pre-split in a per-frame table) with 2-D TMA loads (no multicast); warp 9 allocates TMEM
// and one of its lanes issues the MMAs.  Stages are handed over with mbarriers; every wait
// is bounded and raises TRJ_DEV_TIMEOUT instead of hanging.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <vector>

#include "sq_plan.cuh"

namespace {

constexpr int kProducerWarps = 8;
constexpr int kProducers = kProducerWarps * 32;
constexpr int kTcThreads = kProducers + 64;
constexpr int kStageSlots = 32;            // atoms per stage: K = 64 bf16 = one 128-byte swizzle row
constexpr int kATile = 128 * 128;          // bytes of one 128 x 64 bf16 operand tile
constexpr int kTabEntries = kTcTileNx + kTcTileNy;  // 24 phase factors per atom per stage
constexpr int kMaxStages = 4;

struct TcTile {
    int nx0, ny0, ncols, brow;  // brow: first table row (2*(nz0 - nz_min))
    int64_t acc_off;            // doubles: offset of this tile's [ncols][128] block in a chunk's slice
};

struct TcChunk {
    int species;
    int slot0, slot1;  // [slot0, slot1), multiples of kStageSlots
};

struct TcParams {
    const TcTile* tiles;
    const TcChunk* chunks;
    const uint2* slot_uv;   // (ux, uy) per padded atom slot
    double* part;           // [chunk][acc_stride]
    int64_t acc_stride;
    int nstages;
    int flush_stages;
    int stage_bytes;
    unsigned* status;
};

struct TcState {
    int nz_min = 0, table_rows = 0;
    int64_t total_slots = 0;
    std::vector<int64_t> pad_off;  // nsp+1 padded slot offsets
    std::vector<TcChunk> chunks;
    std::vector<int> chunk_of_species_begin;  // nsp+1
    TcTile* tiles_dev = nullptr;
    TcChunk* chunks_dev = nullptr;
    int64_t* pad_off_dev = nullptr;
    int32_t* chunk_begin_dev = nullptr;
    __nv_bfloat16* tab_hi = nullptr;
    __nv_bfloat16* tab_lo = nullptr;
    uint2* slot_uv = nullptr;
    double* part = nullptr;
    int64_t acc_stride = 0;
    CUtensorMap map_hi, map_lo;
    int nstages = 2, stage_bytes = 0, smem_bytes = 0, max_cols = 0;
    int flush_stages = 32;
};

// ---- PTX wrappers ----------------------------------------------------------

__device__ __forceinline__ void named_bar(int id, int n) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// Barrier `id` over n threads that also returns whether any participant passed pred = true,
// so a group leaves a loop together (a plain named barrier has no timeout).
__device__ __forceinline__ bool bar_any(int id, int n, bool pred) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id), "r"(n)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(trj_smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(trj_smem_addr(bar))
        : "memory");
}

// K-major operand in the 128-byte swizzle: 8-row groups of 1024 bytes (SBO), version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t smem_addr) {
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;              // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;    // stride byte offset: next 8-row group
    d |= (uint64_t)1 << 46;              // descriptor version
    d |= (uint64_t)2 << 61;              // 128-byte swizzle
    return d;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     trj_smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t bf2_bits(__nv_bfloat162 v) { return *reinterpret_cast<uint32_t*>(&v); }

// hi/lo BF16 split of a pair (one value in each half of the 32-bit word, low half first).
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    float2 hf = __bfloat1622float2(h);
    __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
    hi = bf2_bits(h);
    lo = bf2_bits(l);
}

// e^{i pi f} for the fixed-point phase ph (f = ph / 2^31 in [-1, 1)).
__device__ __forceinline__ float2 phase_factor(unsigned ph) {
    float s, c;
    sincospif(__int2float_rn((int)ph) * 4.656612873077393e-10f, &s, &c);
    return make_float2(c, s);
}

// ---- per-frame table: Z phases split into the B operand rows, slot (ux, uy) ----

__global__ void tc_table_kernel(const uint4* __restrict__ phase, const int64_t* __restrict__ sp_off,
                                const int64_t* __restrict__ pad_off, int nsp, int64_t total_slots, int nz_min,
                                int nz_count, int table_rows, int64_t kdim, __nv_bfloat16* __restrict__ tab_hi,
                                __nv_bfloat16* __restrict__ tab_lo, uint2* __restrict__ slot_uv) {
    int64_t slot = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= total_slots) return;
    int a = 0;
    while (a + 1 < nsp && slot >= pad_off[a + 1]) ++a;
    int64_t local = slot - pad_off[a];
    bool real = local < sp_off[a + 1] - sp_off[a];
    uint4 u = real ? phase[sp_off[a] + local] : make_uint4(0u, 0u, 0u, 0u);
    if (blockIdx.y == 0) slot_uv[slot] = make_uint2(u.x, u.y);
    uint32_t* hi = reinterpret_cast<uint32_t*>(tab_hi);
    uint32_t* lo = reinterpret_cast<uint32_t*>(tab_lo);
    for (int t = blockIdx.y; t < table_rows / 2; t += gridDim.y) {
        uint32_t h0 = 0u, l0 = 0u, h1 = 0u, l1 = 0u;
        if (real && t < nz_count) {
            float2 z = phase_factor((unsigned)(nz_min + t) * u.z);
            split2(z.x, -z.y, h0, l0);  // row 2t   (Re out): K(2j) = zr, K(2j+1) = -zi
            split2(z.y, z.x, h1, l1);   // row 2t+1 (Im out): K(2j) = zi, K(2j+1) = zr
        }
        int64_t w0 = (int64_t)(2 * t) * (kdim / 2) + slot;
        int64_t w1 = (int64_t)(2 * t + 1) * (kdim / 2) + slot;
        hi[w0] = h0;
        lo[w0] = l0;
        hi[w1] = h1;
        lo[w1] = l1;
    }
}

// ---- the contraction kernel ------------------------------------------------

__global__ void __launch_bounds__(kTcThreads, 1)
    sq_tc_kernel(const __grid_constant__ CUtensorMap map_hi, const __grid_constant__ CUtensorMap map_lo,
                 TcParams p) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    __shared__ __align__(8) uint64_t full_a[kMaxStages], full_b[kMaxStages], empty[kMaxStages];
    __shared__ __align__(8) uint64_t acc_full, acc_empty;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag_s;
    volatile int& abort_flag = abort_flag_s;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const TcTile T = p.tiles[blockIdx.x];
    const TcChunk C = p.chunks[blockIdx.y];
    const int ncols = T.ncols;
    const int NS = p.nstages;
    const int nst = (C.slot1 - C.slot0) / kStageSlots;
    const int F = p.flush_stages;
    const int nflush = (nst + F - 1) / F;
    float2* tab = reinterpret_cast<float2*>(smem + (size_t)NS * p.stage_bytes);  // [32][24]
    const uint32_t tmem_cols = ncols <= 32 ? 32u : ncols <= 64 ? 64u : ncols <= 128 ? 128u : 256u;

    if (tid == 0) {
        abort_flag = 0;
        for (int s = 0; s < NS; ++s) {
            trj_mbar_init(&full_a[s], kProducerWarps);
            trj_mbar_init(&full_b[s], 1);
            trj_mbar_init(&empty[s], 1);
        }
        trj_mbar_init(&acc_full, 1);
        trj_mbar_init(&acc_empty, kProducerWarps);
        trj_fence_mbar_init();
    }
    if (warp == 9) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         trj_smem_addr(&tmem_slot)),
                     "r"(tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (warp == 8) {
        // ---- B operand: TMA loads of the Z-phase table (hi and lo), 16 rows per load ----
        if (lane == 0 && nst > 0) {
            const unsigned bytes = (unsigned)(2 * ncols * 128);
            for (int s = 0; s < nst; ++s) {
                const int slot = s % NS;
                if (!trj_mbar_wait(&empty[slot], ((s / NS) & 1) ^ 1)) {
                    trj_raise(p.status, TRJ_DEV_TIMEOUT);
                    abort_flag = 1;
                    break;
                }
                uint8_t* bh = smem + (size_t)slot * p.stage_bytes + 2 * kATile;
                uint8_t* bl = bh + ncols * 128;
                trj_mbar_arrive_expect_tx(&full_b[slot], bytes);
                const int k0 = 2 * (C.slot0 + s * kStageSlots);
                for (int r = 0; r < ncols / 16; ++r) {
                    tma_load_2d(bh + r * 2048, &map_hi, k0, T.brow + 16 * r, &full_b[slot]);
                    tma_load_2d(bl + r * 2048, &map_lo, k0, T.brow + 16 * r, &full_b[slot]);
                }
            }
        }
    } else if (warp == 9) {
        // ---- MMA issue: one lane ----
        if (lane == 0 && nst > 0) {
            const uint32_t idesc = (1u << 4)                    // D: F32
                                   | (1u << 7) | (1u << 10)     // A, B: BF16
                                   | ((uint32_t)(ncols >> 3) << 17)
                                   | ((uint32_t)(128 >> 4) << 24);
            int f = 0;
            for (int s = 0; s < nst && !abort_flag; ++s) {
                const int slot = s % NS;
                const unsigned par = (s / NS) & 1;
                const bool first = (s % F) == 0;
                if (first && s > 0) {
                    if (!trj_mbar_wait(&acc_empty, (f - 1) & 1)) {
                        trj_raise(p.status, TRJ_DEV_TIMEOUT);
                        abort_flag = 1;
                        break;
                    }
                }
                if (!trj_mbar_wait(&full_a[slot], par) || !trj_mbar_wait(&full_b[slot], par)) {
                    trj_raise(p.status, TRJ_DEV_TIMEOUT);
                    abort_flag = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t base = trj_smem_addr(smem + (size_t)slot * p.stage_bytes);
                const uint32_t ahi = base, alo = base + kATile, bhi = base + 2 * kATile,
                               blo = bhi + ncols * 128;
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    const uint32_t o = kk * 32;  // 16 bf16 along K
                    mma_bf16(tmem, sw128_desc(ahi + o), sw128_desc(bhi + o), idesc, (first && kk == 0) ? 0u : 1u);
                    mma_bf16(tmem, sw128_desc(ahi + o), sw128_desc(blo + o), idesc, 1u);
                    mma_bf16(tmem, sw128_desc(alo + o), sw128_desc(bhi + o), idesc, 1u);
                }
                mma_commit(&empty[slot]);
                if ((s + 1) % F == 0 || s == nst - 1) {
                    mma_commit(&acc_full);
                    ++f;
                }
            }
        }
    } else {
        // ---- A operand producers (warps 0-7), then TMEM drain ----
        const int ptid = tid;  // 0..255
        const int m = ptid & 127, half = ptid >> 7;
        const int nxl = m & 15, nyl = m >> 4;
        const uint32_t rowoff = (uint32_t)((m >> 3) * 1024 + (m & 7) * 128);
        int f = 0;
        for (int s = 0; s < nst; ++s) {
            const int slot = s % NS;
            const int sbase = C.slot0 + s * kStageSlots;
            named_bar(1, kProducers);  // previous stage's table reads are done
            for (int q = ptid; q < kStageSlots * kTabEntries; q += kProducers) {
                const int j = q / kTabEntries, e = q % kTabEntries;
                const uint2 uv = p.slot_uv[sbase + j];
                const unsigned ph = e < kTcTileNx ? (unsigned)(T.nx0 + e) * uv.x
                                                  : (unsigned)(T.ny0 + e - kTcTileNx) * uv.y;
                tab[q] = phase_factor(ph);
            }
            named_bar(1, kProducers);
            const bool ok = trj_mbar_wait(&empty[slot], ((s / NS) & 1) ^ 1);
            if (bar_any(1, kProducers, !ok || abort_flag)) {
                trj_raise(p.status, TRJ_DEV_TIMEOUT);
                abort_flag = 1;
                break;
            }
            uint8_t* ahi = smem + (size_t)slot * p.stage_bytes;
            uint8_t* alo = ahi + kATile;
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
                const int c = half * 4 + cc;  // 16-byte chunk = 4 atoms along K
                uint32_t hw[4], lw[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int j = c * 4 + q;
                    const float2 x = tab[j * kTabEntries + nxl];
                    const float2 y = tab[j * kTabEntries + kTcTileNx + nyl];
                    const float ar = x.x * y.x - x.y * y.y;
                    const float ai = x.x * y.y + x.y * y.x;
                    split2(ar, ai, hw[q], lw[q]);
                }
                const uint32_t off = rowoff + (uint32_t)((c ^ (m & 7)) << 4);
                *reinterpret_cast<uint4*>(ahi + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
                *reinterpret_cast<uint4*>(alo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
            }
            fence_proxy_async();
            __syncwarp();
            if (lane == 0) trj_mbar_arrive(&full_a[slot]);
            if ((s + 1) % F == 0 || s == nst - 1) {
                // drain the FP32 accumulator into this CTA's FP64 block
                const bool okf = trj_mbar_wait(&acc_full, f & 1);
                if (bar_any(1, kProducers, !okf)) {
                    trj_raise(p.status, TRJ_DEV_TIMEOUT);
                    abort_flag = 1;
                    break;
                }
                tc_fence_after();
                const int q4 = warp & 3, h2 = warp >> 2;
                const int row = 32 * q4 + lane;
                const int c0 = h2 * (ncols / 2), c1 = c0 + ncols / 2;
                double* dst = p.part + (int64_t)blockIdx.y * p.acc_stride + T.acc_off;
                for (int c = c0; c < c1; c += 8) {
                    uint32_t r[8];
                    tmem_ld8(tmem + ((uint32_t)(32 * q4) << 16) + (uint32_t)c, r);
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        double* d = dst + (int64_t)(c + i) * 128 + row;
                        const double v = (double)__uint_as_float(r[i]);
                        if (f == 0) *d = v;
                        else *d += v;
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) trj_mbar_arrive(&acc_empty);
                ++f;
            }
        }
        (void)nflush;
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 9) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols)
                     : "memory");
    }
}

// tc_out[tile][a][col][row] = sum over species a's chunks (fixed order) of the FP64 blocks.
__global__ void tc_reduce_kernel(const double* __restrict__ part, int64_t acc_stride, const TcTile* __restrict__ tiles,
                                 const SqTile* __restrict__ stiles, const int32_t* __restrict__ chunk_begin, int nsp,
                                 double* __restrict__ out) {
    const int t = blockIdx.x;
    const TcTile T = tiles[t];
    const int64_t n = (int64_t)T.ncols * 128;
    for (int a = 0; a < nsp; ++a) {
        const int k0 = chunk_begin[a], k1 = chunk_begin[a + 1];
        for (int64_t e = threadIdx.x; e < n; e += blockDim.x) {
            double s = 0.0;
            for (int k = k0; k < k1; ++k) s += part[(int64_t)k * acc_stride + T.acc_off + e];
            out[stiles[t].out_off + (int64_t)a * n + e] = s;
        }
    }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn get_encode() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(ptr);
    }
    return fn;
}

int encode_map(trj_ctx* ctx, CUtensorMap* map, void* base, int64_t kdim, int rows) {
    EncodeTiledFn enc = get_encode();
    if (!enc) return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[2] = {(cuuint64_t)kdim, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)kdim * 2};
    cuuint32_t box[2] = {64, 16};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return trj_fail(ctx, TRJ_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return TRJ_OK;
}

}  // namespace

void trj_sq_tc_release(trj_sq_plan* plan) {
    TcState* st = reinterpret_cast<TcState*>(plan->tc_state);
    if (!st) return;
    void* ptrs[] = {st->tiles_dev, st->chunks_dev, st->pad_off_dev, st->chunk_begin_dev,
                    st->tab_hi, st->tab_lo, st->slot_uv, st->part};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    delete st;
    plan->tc_state = nullptr;
}

int trj_sq_tc_prepare(trj_sq_plan* plan) {
    trj_ctx* ctx = plan->ctx;
    if (plan->tiles.empty()) return TRJ_OK;
    TcState* st = new TcState();
    plan->tc_state = st;
    const int nsp = plan->nsp;
    // padded atom slots per species
    st->pad_off.assign(nsp + 1, 0);
    for (int a = 0; a < nsp; ++a)
        st->pad_off[a + 1] = st->pad_off[a] + (plan->species_counts[a] + kStageSlots - 1) / kStageSlots * kStageSlots;
    st->total_slots = std::max<int64_t>(st->pad_off[nsp], kStageSlots);
    if (2 * st->total_slots > (int64_t)INT32_MAX) return trj_fail(ctx, TRJ_ERR_CAPACITY, "tensor path: frame too large");
    // table rows and tiles
    int nz_min = plan->tiles[0].nz0, nz_max = nz_min;
    for (const SqTile& t : plan->tiles) {
        nz_min = std::min(nz_min, t.nz0);
        nz_max = std::max(nz_max, t.nz0 + t.ncols / 2 - 1);
    }
    st->nz_min = nz_min;
    st->table_rows = 2 * (nz_max - nz_min + 1);
    std::vector<TcTile> tt(plan->tiles.size());
    int64_t acc = 0;
    for (size_t i = 0; i < plan->tiles.size(); ++i) {
        const SqTile& s = plan->tiles[i];
        tt[i] = TcTile{s.nx0, s.ny0, s.ncols, 2 * (s.nz0 - nz_min), acc};
        acc += (int64_t)s.ncols * 128;
        st->max_cols = std::max(st->max_cols, s.ncols);
    }
    st->acc_stride = acc;
    // chunks: each species' slots split so that tiles x chunks covers the GPU about twice
    const int64_t ntiles = (int64_t)tt.size();
    const int64_t target_chunks = std::max<int64_t>(nsp, (2 * ctx->sm_count + ntiles - 1) / ntiles);
    const int64_t total_real = std::max<int64_t>(1, plan->n_total);
    st->chunk_begin_dev = nullptr;
    st->chunk_of_species_begin.assign(nsp + 1, 0);
    for (int a = 0; a < nsp; ++a) {
        st->chunk_of_species_begin[a] = (int)st->chunks.size();
        const int64_t slots = st->pad_off[a + 1] - st->pad_off[a];
        const int64_t stages = slots / kStageSlots;
        if (stages == 0) continue;
        int64_t k = std::max<int64_t>(1, (target_chunks * plan->species_counts[a] + total_real - 1) / total_real);
        k = std::min<int64_t>(k, stages);
        for (int64_t i = 0; i < k; ++i) {
            const int64_t s0 = stages * i / k, s1 = stages * (i + 1) / k;
            if (s1 > s0)
                st->chunks.push_back(TcChunk{a, (int)(st->pad_off[a] + s0 * kStageSlots),
                                             (int)(st->pad_off[a] + s1 * kStageSlots)});
        }
    }
    st->chunk_of_species_begin[nsp] = (int)st->chunks.size();
    if (st->chunks.empty()) return TRJ_OK;
    // shared memory: stages of (A hi, A lo, B hi, B lo) + the X/Y phase table
    st->stage_bytes = 2 * kATile + 2 * st->max_cols * 128;
    const int table_bytes = kStageSlots * kTabEntries * (int)sizeof(float2);
    const int avail = (int)ctx->smem_optin - 1024 - table_bytes - 512;
    st->nstages = std::min(kMaxStages, avail / st->stage_bytes);
    if (st->nstages < 2) return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "tensor path: tile too wide for shared memory");
    st->smem_bytes = st->nstages * st->stage_bytes + table_bytes + 1024;

    const int64_t kdim = 2 * st->total_slots;
    size_t tab_bytes = (size_t)st->table_rows * (size_t)kdim * sizeof(__nv_bfloat16);
    size_t part_bytes = sizeof(double) * (size_t)st->acc_stride * st->chunks.size();
    std::vector<int32_t> cb(st->chunk_of_species_begin.begin(), st->chunk_of_species_begin.end());
    if (cudaMalloc(&st->tab_hi, tab_bytes) != cudaSuccess || cudaMalloc(&st->tab_lo, tab_bytes) != cudaSuccess ||
        cudaMalloc(&st->slot_uv, sizeof(uint2) * st->total_slots) != cudaSuccess ||
        cudaMalloc(&st->part, part_bytes) != cudaSuccess ||
        cudaMalloc(&st->tiles_dev, sizeof(TcTile) * tt.size()) != cudaSuccess ||
        cudaMalloc(&st->chunks_dev, sizeof(TcChunk) * st->chunks.size()) != cudaSuccess ||
        cudaMalloc(&st->pad_off_dev, sizeof(int64_t) * (nsp + 1)) != cudaSuccess ||
        cudaMalloc(&st->chunk_begin_dev, sizeof(int32_t) * (nsp + 1)) != cudaSuccess)
        return trj_fail(ctx, TRJ_ERR_NOMEM, "tensor path: %zu bytes of tables", 2 * tab_bytes + part_bytes);
    cudaMemcpy(st->tiles_dev, tt.data(), sizeof(TcTile) * tt.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(st->chunks_dev, st->chunks.data(), sizeof(TcChunk) * st->chunks.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(st->pad_off_dev, st->pad_off.data(), sizeof(int64_t) * (nsp + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(st->chunk_begin_dev, cb.data(), sizeof(int32_t) * (nsp + 1), cudaMemcpyHostToDevice);
    plan->scratch_bytes += (int64_t)(2 * tab_bytes + part_bytes + sizeof(uint2) * st->total_slots);
    int rc = encode_map(ctx, &st->map_hi, st->tab_hi, kdim, st->table_rows);
    if (rc == TRJ_OK) rc = encode_map(ctx, &st->map_lo, st->tab_lo, kdim, st->table_rows);
    if (rc != TRJ_OK) return rc;
    TRJ_CUDA_TRY(ctx, cudaFuncSetAttribute(sq_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           st->smem_bytes));
    return TRJ_OK;
}

int trj_sq_tc_run(trj_sq_plan* plan, const float box[3], cudaStream_t s) {
    (void)box;
    trj_ctx* ctx = plan->ctx;
    TcState* st = reinterpret_cast<TcState*>(plan->tc_state);
    if (!st || !st->tab_hi)
        return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "tensor-core S(Q) path was not prepared for this plan");
    const int64_t kdim = 2 * st->total_slots;
    const int nz_count = st->table_rows / 2;
    dim3 tg((unsigned)((st->total_slots + 255) / 256), (unsigned)std::min(nz_count, 64));
    tc_table_kernel<<<tg, 256, 0, s>>>(plan->phase_dev, plan->species_off_dev, st->pad_off_dev, plan->nsp,
                                       st->total_slots, st->nz_min, nz_count, st->table_rows, kdim, st->tab_hi,
                                       st->tab_lo, st->slot_uv);
    TcParams P;
    P.tiles = st->tiles_dev;
    P.chunks = st->chunks_dev;
    P.slot_uv = st->slot_uv;
    P.part = st->part;
    P.acc_stride = st->acc_stride;
    P.nstages = st->nstages;
    P.flush_stages = st->flush_stages;
    P.stage_bytes = st->stage_bytes;
    P.status = ctx->status_dev;
    dim3 grid((unsigned)plan->tiles.size(), (unsigned)st->chunks.size());
    plan->timer.begin(ctx, s);
    sq_tc_kernel<<<grid, kTcThreads, st->smem_bytes, s>>>(st->map_hi, st->map_lo, P);
    plan->timer.end(ctx, s);
    tc_reduce_kernel<<<(unsigned)plan->tiles.size(), 256, 0, s>>>(st->part, st->acc_stride, st->tiles_dev,
                                                                  plan->tiles_dev, st->chunk_begin_dev, plan->nsp,
                                                                  plan->tc_out_dev);
    ctx->launches += 3;
    TRJ_CUDA_TRY(ctx, cudaGetLastError());
    return TRJ_OK;
}
