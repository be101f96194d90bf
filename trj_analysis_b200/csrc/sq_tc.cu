// sq_tc.cu -- tensor-core S(Q): rho_a(k) for a compact k-region as a BF16 tcgen05 contraction.
//
// For lattice vectors k = 2 pi (nx/Lx, ny/Ly, nz/Lz) the phase factor separates:
//   e^{i k.r_j} = X_j[nx] * Y_j[ny] * Z_j[nz],   X_j[n] = e^{2 pi i n x_j/Lx}, ...
// so for a tile of 128 (nx, ny) rows (16 nx x 8 ny) and a run of nz values,
//   rho(nx, ny, nz) = sum_j A[(nx,ny), j] * Z_j[nz],   A = X*Y,
// a complex GEMM with the atoms as the contraction dimension.  It runs as a real GEMM:
//   K index 2j = Re, 2j+1 = Im of atom j;  B columns 2t (Re out) = (zr, -zi), 2t+1 (Im out) = (zi, zr).
// Each factor v is split v = hi + lo with hi = bf16(v), lo = bf16(v - hi); the product keeps
// hi*hi + hi*lo + lo*hi (three tcgen05.mma kind::f16 per K-step into one FP32 TMEM accumulator).
//
// Operands: A is built by the producer warps straight into tensor memory (the tcgen05.mma form
// with A in TMEM), in two alternating half-stage buffers of 16 atoms, so shared-memory bandwidth
// goes to the B operand only.  B (the split Z factors) is a per-frame table, blocked by 32-atom stage
// ([stage][row][32 atoms x (re, im)], so one stage's rows are contiguous), read with 2-D TMA loads
// (128-byte swizzle, no multicast) through a ring of 32-atom stages; each stage also carries the
// atoms' x/y phases, from which the producers evaluate the X and Y factors of the tile in shared
// memory before forming the products.  Tiles are up to 224 columns wide: one tcgen05.mma costs at
// least ~90 cycles whatever its width, so wide tiles keep the tensor pipe busy.
//
// Accumulation: the tensor core's FP32 accumulation is biased (the error of a run grows linearly
// with its length), so every F stages (F*32 atoms, 256 by default) the accumulator is drained: the
// epilogue warps add it with round-to-nearest CUDA-core adds into an FP32 running sum kept in
// TMEM, and the last drain of a work item stores that sum once, in FP64, to global memory.  The
// blocks of one species are then summed in FP64 in a fixed order.
//
// Phases: every coordinate is the 32-bit fixed-point fraction u = (x/L mod 1) 2^32 (from FP64);
// n*u mod 2^32 in integer arithmetic is exact, and sincospif of the reduced fraction gives each
// factor at FP32 accuracy.
//
// Work item = (tile, chunk of one species' atoms).  Persistent CTAs walk their items chunk-major.
// Roles per CTA (704 threads), handing stages to each other through mbarriers only: warps 8-11
// evaluate the X/Y factors of a stage into one of two shared-memory buffers; warps 0-7 form the
// products, split them and store them into the A buffers in TMEM (the two warps of one TMEM lane
// quarter split a half-stage's 16 atoms); warps 12-19 drain the accumulator (two warps per lane
// quarter, alternating 16-column chunks); warp 20 issues the TMA loads; warp 21 allocates TMEM and
// one of its lanes issues the MMAs.  Each role runs at its own pace: a warp arrives on a barrier and
// moves on (two forms that tied the roles closer were slower at c3: the builders evaluating the
// factors themselves and issuing the MMAs, 16.2 ms, and the builders issuing the MMAs after a named
// barrier per half-stage, 13.5 ms, against 10.9 ms).  Every mbarrier wait is bounded and raises TRJ_DEV_TIMEOUT instead of hanging.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <vector>

#include "sq_plan.cuh"

namespace {

// Builders: two warps per TMEM lane quarter, each taking 8 atoms of a half-stage.  Measured at c3
// against other layouts of the same roles: four warps per quarter (4 atoms each) 11.46 ms, against
// 10.88 ms for two.
constexpr int kBuildWarps = 8;                     // warps 0-7: A products into TMEM
constexpr int kXyWarps = 4;                        // warps 8-11: X/Y factors into shared memory
constexpr int kEpiWarps = 8;                       // warps 12-19: accumulator drains
constexpr int kXyWarp0 = kBuildWarps;
constexpr int kEpiWarp0 = kXyWarp0 + kXyWarps;
constexpr int kTmaWarp = kEpiWarp0 + kEpiWarps;    // 20
constexpr int kMmaWarp = kTmaWarp + 1;             // 21
constexpr int kTcThreads = (kMmaWarp + 1) * 32;    // 704 (CTA-pair form)
// One-CTA form: the X/Y factors come from per-frame tables through their own stage ring, so it has
// no factor warps; the FP32 running sum of the drains lives in the epilogue warps' registers, which
// leaves TMEM to the accumulator and a deep ring of A buffers.
constexpr int k1EpiWarps = 16;                     // warps 8-23: drains, four warps per lane quarter
constexpr int k1EpiWarp0 = kBuildWarps;
constexpr int k1TmaWarp = k1EpiWarp0 + k1EpiWarps;  // 24: B rows
constexpr int k1XyWarp = k1TmaWarp + 1;             // 25: X/Y factor blocks
constexpr int k1MmaWarp = k1XyWarp + 1;             // 26
constexpr int k1Threads = (k1MmaWarp + 1) * 32;     // 864
// Running sum of an epilogue thread: 8-column chunks cg, cg + 4, ..., the first k1RegChunks of them in
// registers, the next (columns 192-223, tiles wider than 192 columns only) in shared memory
// [warp][8][32 lanes] (16 KB), so that the epilogue fits the 72 registers a thread of 864 has.
constexpr int k1RegChunks = 6;
constexpr int k1TailCol = 8 * 4 * k1RegChunks;      // 192
constexpr int k1TailBytes = k1EpiWarps * 8 * 32 * 4;  // 16 KB
constexpr int k1MaxABufs = 9;                       // A half-stage buffers of 32 TMEM columns
constexpr int kXyStages = 6;                        // X/Y factor-block ring
static_assert(k1TailCol + 32 >= 224, "running-sum chunks cover the widest tile");
constexpr int kStageSlots = 32;  // atoms per stage: K = 64 bf16 = one 128-byte swizzle row of B
constexpr int kBuildGroups = kBuildWarps / 4;      // builder warps per lane quarter
constexpr int kHalfAtoms = kStageSlots / 2 / kBuildGroups;  // atoms of a half-stage per builder warp
static_assert(kBuildWarps % 4 == 0 && kHalfAtoms % 4 == 0, "builder layout");
// X/Y factor rows: 32 atoms as (re, im) plus 2 pad entries, so that rows start 272 bytes (68 banks)
// apart and the 16-byte loads of eight lanes on eight different rows fall in different banks.
constexpr int kXyRow = kStageSlots + 2;
constexpr int kXBytes = kXyRow * kTcTileNx * 8;  // X factors [16 nx][kXyRow] as (xr, xi)
constexpr int kYBytes = kXyRow * kTcTileNy * 8;  // Y factors [8 ny][kXyRow] as (yr, yi)
constexpr int kXyBytes = kXBytes + kYBytes;           // one of the two X/Y buffers
constexpr int kUxyBytes = kStageSlots * 8;            // 32 atoms x (ux, uy)
// Factor blocks of one stage in the one-CTA form: [16 atom pairs][16 nx (8 ny)] x (re, im) of the pair's
// two atoms, the order in which the builders read them.
constexpr int kXBlockBytes = kStageSlots / 2 * kTcTileNx * 16;  // 4096
constexpr int kYBlockBytes = kStageSlots / 2 * kTcTileNy * 16;  // 2048
constexpr int kMaxStages = 8;
constexpr int kChunkAtoms = 12288;  // atom slots per chunk: the Z-table rows of one chunk are ~10 MB
constexpr int kMaxTileCols = 224;
// TMEM columns of the one-CTA form (512 allocated): the accumulator at 0 (bmax columns, the widest
// tile), then from the next multiple of 32 as many A half-stage buffers of 32 columns (16 of packed
// bf16 pairs for hi, then 16 for lo) as fit, up to k1MaxABufs: 9 for every bmax <= 224.
constexpr uint32_t kTmemCols = 512;
// CTA-pair form: accumulator at 0, four full-stage A buffers (32 columns hi, 32 lo) from 224; its
// FP32 running sum lives in shared memory.
constexpr uint32_t kPairACol = 224;
constexpr int kPairABufs = 4;
static_assert(kPairACol + 64 * kPairABufs <= kTmemCols, "pair TMEM layout");
static_assert(kTcRows == 128, "one TMEM lane per A row");
static_assert(kMaxTileCols <= kTcMaxCols, "tile width");

struct TcTile {
    int nx0, ny0, ncols, brow;  // brow: first Z-table row (2*(nz0 - nz_min))
    int64_t acc_off;            // doubles: offset of this tile's [ncols][128] block in a chunk's slice
};

struct TcChunk {
    int species;
    int slot0, slot1;  // [slot0, slot1), multiples of kStageSlots
};

struct TcParams {
    const TcTile* tiles;
    const TcChunk* chunks;
    const int32_t* cta_items;  // item ids (chunk * ntiles + tile) of every CTA, concatenated
    const int32_t* cta_off;    // gridDim.x + 1 offsets into cta_items
    const uint2* uxy;          // per slot: x and y phase fractions
    float* part;               // [chunk][acc_stride]: each item's FP32 running sum (exact in FP64)
    int64_t acc_stride;
    int ntiles, nchunks;
    int nstages;
    int flush_stages;
    int stage_bytes;  // one B stage: hi then lo rows
    int bmax;  // B rows of a stage buffer
    int table_rows;  // Z-table rows per 32-slot block
    uint32_t a_col;  // TMEM column of the first A buffer
    int nabuf;       // A half-stage buffers
    const float4* xtab;       // X factor blocks [stage][nx block][pair][16]
    const float4* ytab;       // Y factor blocks [stage][ny block][pair][8]
    int nxb, nyb, nx0min, ny0min;
    unsigned* status;
};

// Two tiles sharing one B (the union of their nz spans): the leader CTA of a cluster holds the first
// tile's 128 rows of the M = 256 accumulator, the peer the second's; each CTA holds half of B's rows.
struct TcPairDev {
    int tile[2];   // tile of the leader / the peer, -1 for none
    int coff[2];   // accumulator column of each tile's first own column
    int ncols;     // N of the pair: multiple of 32, <= kMaxTileCols
    int brow;      // first Z-table row of the pair's B
    int nx0[2], ny0[2];
};

struct Tc2Params {
    const TcTile* tiles;
    const TcPairDev* pairs;
    const TcChunk* chunks;
    const int32_t* cl_items;  // item ids (chunk * npairs + pair) of every cluster, concatenated
    const int32_t* cl_off;    // nclusters + 1 offsets into cl_items
    const uint2* uxy;
    float* part;
    int64_t acc_stride;
    int npairs, nchunks;
    int nstages;
    int flush_stages;
    int stage_bytes;
    int bhalf;  // B rows per CTA of a stage buffer
    int table_rows;  // Z-table rows per 32-slot block
    unsigned* status;
};

struct TcState {
    int nz_min = 0, table_rows = 0;
    int64_t total_slots = 0;
    std::vector<int64_t> pad_off;  // nsp+1 padded slot offsets
    std::vector<TcChunk> chunks;
    std::vector<int> chunk_of_species_begin;  // nsp+1
    TcTile* tiles_dev = nullptr;
    int32_t* sched_dev = nullptr;  // [grid + 1 offsets][items]
    TcChunk* chunks_dev = nullptr;
    int64_t* pad_off_dev = nullptr;  // nsp+1 offsets, then nsp slot -> atom multipliers
    int32_t* chunk_begin_dev = nullptr;
    __nv_bfloat16* tab_hi = nullptr;
    __nv_bfloat16* tab_lo = nullptr;
    uint2* uxy = nullptr;
    float4* xtab = nullptr;  // X/Y factor blocks of the one-CTA form
    float4* ytab = nullptr;
    int nxb = 0, nyb = 0, nx0min = 0, ny0min = 0;
    float* part = nullptr;  // per-item FP32 sums, summed per species in FP64 by tc_reduce_kernel
    int64_t acc_stride = 0;
    CUtensorMap map_hi, map_lo, map_hi64, map_lo64;  // 16-row and 64-row boxes
    int nstages = 2, stage_bytes = 0, smem_bytes = 0, bmax = 0;
    int nabuf = 2;  // A half-stage buffers in TMEM
    int a_col = 0;  // TMEM column of the first A buffer
    int flush_stages = 8;  // 256 atoms per FP32 tensor-core run between drains
    int grid = 0;
    // CTA-pair (cta_group::2) form
    int pairs_ok = 0, use_pairs = 0;  // pair form on request (slower than one CTA per tile at c3)
    int npairs = 0, grid2 = 0, nstages2 = 2, stage_bytes2 = 0, smem_bytes2 = 0, bhalf = 0;
    TcPairDev* pairs_dev = nullptr;
    int32_t* sched2_dev = nullptr;
};

// ---- PTX wrappers ----------------------------------------------------------

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
    d |= (uint64_t)1 << 16;            // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;  // stride byte offset: next 8-row group
    d |= (uint64_t)1 << 46;            // descriptor version
    d |= (uint64_t)2 << 61;            // 128-byte swizzle
    return d;
}

// D (TMEM) += A (TMEM, 128 lanes x 16 bf16) * B (shared-memory descriptor)^T.
__device__ __forceinline__ void mma_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(tmem_d),
        "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accum)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     trj_smem_addr(bar))
                 : "memory");
}

// tcgen05.ld without the wait, so that several loads are in flight before one tmem_wait_ld.
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld8_nowait(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
        "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}

__device__ __forceinline__ void tmem_st4(uint32_t taddr, const uint32_t (&r)[4]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), "r"(r[0]), "r"(r[1]),
                 "r"(r[2]), "r"(r[3])
                 : "memory");
}

template <int NJ>
__device__ __forceinline__ void tmem_st_cols(uint32_t taddr, const uint32_t (&r)[NJ]) {
    if constexpr (NJ == 8) tmem_st8(taddr, r);
    else tmem_st4(taddr, r);
}

__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t bf2_bits(__nv_bfloat162 v) { return *reinterpret_cast<uint32_t*>(&v); }

// e^{i pi f} for the fixed-point phase ph (f = ph / 2^31 in [-1, 1)).
__device__ __forceinline__ float2 phase_factor(unsigned ph) {
    float s, c;
    sincospif(__int2float_rn((int)ph) * 4.656612873077393e-10f, &s, &c);
    return make_float2(c, s);
}

// A = X * Y: (ar, ai) = (xr yr - xi yi, xr yi + xi yr), each rounded once after the first product,
// then the hi/lo BF16 split of (ar, ai) (low half of each word: ar).
__device__ __forceinline__ void product_split(float xr, float xi, float yr, float yi, uint32_t& hi, uint32_t& lo) {
    const float ar = __fmaf_rn(xr, yr, -__fmul_rn(xi, yi));
    const float ai = __fmaf_rn(xr, yi, __fmul_rn(xi, yr));
    const uint32_t h = bf2_bits(__floats2bfloat162_rn(ar, ai));
    const float dr = __fsub_rn(ar, __uint_as_float(h << 16));  // exact: ar minus its 8-bit rounding
    const float di = __fsub_rn(ai, __uint_as_float(h & 0xffff0000u));
    hi = h;
    lo = bf2_bits(__floats2bfloat162_rn(dr, di));
}

// X/Y buffer: X factors [16 nx][kXyRow], then Y factors [8 ny][kXyRow], each (re, im) per atom.
// Consecutive threads take consecutive atoms of one nx (ny): each thread reads its atom's phases once per
// factor, and a warp's stores cover one row.
__device__ __forceinline__ void fill_xy(float2* xs, const uint2* u, int nx0, int ny0, int xt, int nthreads) {
    float2* ys = xs + kTcTileNx * kXyRow;
    for (int e = xt; e < kStageSlots * kTcTileNx; e += nthreads)
        xs[(e >> 5) * kXyRow + (e & 31)] = phase_factor((unsigned)(nx0 + (e >> 5)) * u[e & (kStageSlots - 1)].x);
    for (int e = xt; e < kStageSlots * kTcTileNy; e += nthreads)
        ys[(e >> 5) * kXyRow + (e & 31)] = phase_factor((unsigned)(ny0 + (e >> 5)) * u[e & (kStageSlots - 1)].y);
}

// The hi and lo BF16 pairs of A for row (nxl, nyl) and atoms j0 .. j0 + NJ - 1 of the stage (j0 a
// multiple of 4): every 16-byte load carries two atoms' factors that this lane uses.
template <int NJ>
__device__ __forceinline__ void build_row(const float2* xs, int nxl, int nyl, int j0, uint32_t (&hw)[NJ],
                                          uint32_t (&lw)[NJ]) {
    const float4* xr = reinterpret_cast<const float4*>(xs + nxl * kXyRow + j0);
    const float4* yr = reinterpret_cast<const float4*>(xs + (kTcTileNx + nyl) * kXyRow + j0);
#pragma unroll
    for (int k = 0; k < NJ / 2; ++k) {
        const float4 x = xr[k], y = yr[k];
        product_split(x.x, x.y, y.x, y.y, hw[2 * k], lw[2 * k]);
        product_split(x.z, x.w, y.z, y.w, hw[2 * k + 1], lw[2 * k + 1]);
    }
}

// hi/lo BF16 split of a pair (one value in each half of the 32-bit word, low half first).
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    float2 hf = __bfloat1622float2(h);
    __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
    hi = bf2_bits(h);
    lo = bf2_bits(l);
}

__device__ __forceinline__ bool timed_wait(uint64_t* bar, unsigned parity, unsigned* status) {
    if (trj_mbar_wait(bar, parity)) return true;
    trj_raise(status, TRJ_DEV_TIMEOUT);
    return false;
}

// ---- per-frame table ---------------------------------------------------------
// slot -> atom of the species-padded layout; padding slots carry zero factors.  Within a species
// the slots visit the atoms in the order local * mul[a] mod n_a (mul coprime with n_a, near the
// golden ratio of n_a; mul = pad_off + nsp + 1): packed frames are cell-sorted, so consecutive atoms
// are close in space and, at small k, their phase factors nearly equal.  Scattered, a run of slots
// samples the whole box and its partial sums stay small, which keeps the FP32 accumulation error of
// the tensor cores and of the running sums small compared with rho.
__device__ __forceinline__ bool slot_atom(int64_t slot, const int64_t* pad_off, const int64_t* sp_off, int nsp,
                                          int64_t& atom) {
    int a = 0;
    while (a + 1 < nsp && slot >= pad_off[a + 1]) ++a;
    const int64_t local = slot - pad_off[a];
    const int64_t na = sp_off[a + 1] - sp_off[a];
    if (local >= na) return false;
    atom = sp_off[a] + (int64_t)(((uint64_t)local * (uint64_t)pad_off[nsp + 1 + a]) % (uint64_t)na);  // < 2^62
    return true;
}

// Z factors split into the B operand rows (row 2t: (zr, -zi), row 2t+1: (zi, zr) along K), and the
// x/y phase fractions of every slot (zero for padding slots, whose Z rows are zero).
__global__ void tc_ztable_kernel(const uint4* __restrict__ phase, const int64_t* __restrict__ sp_off,
                                 const int64_t* __restrict__ pad_off, int nsp, int64_t total_slots, int nz_min,
                                 int nz_count, int64_t table_rows, __nv_bfloat16* __restrict__ tab_hi,
                                 __nv_bfloat16* __restrict__ tab_lo, uint2* __restrict__ uxy, int64_t qbase) {
    int64_t slot = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= total_slots) return;
    int64_t atom = 0;
    const bool real = slot_atom(slot, pad_off, sp_off, nsp, atom);
    const uint4 u = real ? phase[atom] : make_uint4(0u, 0u, 0u, 0u);
    if (blockIdx.y == 0) uxy[slot] = make_uint2(u.x, u.y);
    // entries from qbase on belong to the charge species: the Z factor carries the charge
    const float wq = (real && atom >= qbase) ? __uint_as_float(u.w) : 1.0f;
    uint32_t* hi = reinterpret_cast<uint32_t*>(tab_hi);
    uint32_t* lo = reinterpret_cast<uint32_t*>(tab_lo);
    for (int t = blockIdx.y; t < nz_count; t += gridDim.y) {
        uint32_t h0 = 0u, l0 = 0u, h1 = 0u, l1 = 0u;
        if (real) {
            float2 z = phase_factor((unsigned)(nz_min + t) * u.z);
            z.x *= wq;
            z.y *= wq;
            split2(z.x, -z.y, h0, l0);
            split2(z.y, z.x, h1, l1);
        }
        // blocked layout [slot / 32][row][32 slots x (re, im)]: a stage's rows are contiguous
        const int64_t w0 = ((slot / kStageSlots) * table_rows + 2 * t) * kStageSlots + (slot % kStageSlots);
        const int64_t w1 = w0 + kStageSlots;
        hi[w0] = h0;
        lo[w0] = l0;
        hi[w1] = h1;
        lo[w1] = l1;
    }
}

// X and Y factors of every 32-slot stage, per block of 16 nx (8 ny) values of the tiles, in the order
// the builders read them: [stage][block][atom pair][value of the block] x (re, im) of the pair's two
// atoms.  Consecutive threads take consecutive values of one pair: the stores of a warp are contiguous.
__global__ void tc_xytable_kernel(const uint2* __restrict__ uxy, int64_t nstage, int nxb, int nx0min, int nyb,
                                  int ny0min, float4* __restrict__ xtab, float4* __restrict__ ytab) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nxe = nstage * nxb * (kStageSlots / 2) * kTcTileNx;
    const int64_t nye = nstage * nyb * (kStageSlots / 2) * kTcTileNy;
    if (e < nxe) {
        const int v = (int)(e & (kTcTileNx - 1)), pair = (int)((e / kTcTileNx) & (kStageSlots / 2 - 1));
        const int64_t sb = e / (kTcTileNx * kStageSlots / 2);
        const int b = (int)(sb % nxb);
        const int64_t slot = (sb / nxb) * kStageSlots + 2 * pair;
        const unsigned n = (unsigned)(nx0min + kTcTileNx * b + v);
        const float2 f0 = phase_factor(n * uxy[slot].x), f1 = phase_factor(n * uxy[slot + 1].x);
        xtab[e] = make_float4(f0.x, f0.y, f1.x, f1.y);
    } else if (e < nxe + nye) {
        const int64_t f = e - nxe;
        const int v = (int)(f & (kTcTileNy - 1)), pair = (int)((f / kTcTileNy) & (kStageSlots / 2 - 1));
        const int64_t sb = f / (kTcTileNy * kStageSlots / 2);
        const int b = (int)(sb % nyb);
        const int64_t slot = (sb / nyb) * kStageSlots + 2 * pair;
        const unsigned n = (unsigned)(ny0min + kTcTileNy * b + v);
        const float2 f0 = phase_factor(n * uxy[slot].y), f1 = phase_factor(n * uxy[slot + 1].y);
        ytab[f] = make_float4(f0.x, f0.y, f1.x, f1.y);
    }
}

// The hi and lo BF16 pairs of A for row (nxl, nyl) and the 8 atoms of pairs p0 .. p0 + 3 from a stage's
// factor blocks (lanes of one quarter-warp read consecutive 16-byte entries: no bank conflicts).
__device__ __forceinline__ void build_row_tab(const float4* xb, const float4* yb, int nxl, int nyl, int p0,
                                              uint32_t (&hw)[8], uint32_t (&lw)[8]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float4 x = xb[(p0 + k) * kTcTileNx + nxl], y = yb[(p0 + k) * kTcTileNy + nyl];
        product_split(x.x, x.y, y.x, y.y, hw[2 * k], lw[2 * k]);
        product_split(x.z, x.w, y.z, y.w, hw[2 * k + 1], lw[2 * k + 1]);
    }
}

// ---- the contraction kernel ------------------------------------------------

__global__ void __launch_bounds__(k1Threads, 1)
    sq_tc_kernel(const __grid_constant__ CUtensorMap map_hi, const __grid_constant__ CUtensorMap map_lo,
                 const __grid_constant__ CUtensorMap map_hi64, const __grid_constant__ CUtensorMap map_lo64, TcParams p) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    __shared__ __align__(8) uint64_t full_b[kMaxStages], empty_b[kMaxStages], full_xy[kXyStages], empty_xy[kXyStages];
    __shared__ __align__(8) uint64_t full_a[k1MaxABufs], empty_a[k1MaxABufs], acc_full, acc_empty, mma_done;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag_s;
    volatile int& abort_flag = abort_flag_s;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int NS = p.nstages;
    const int NA = p.nabuf;
    const int F = p.flush_stages;
    const int item0 = p.cta_off[blockIdx.x], item1 = p.cta_off[blockIdx.x + 1];
    // shared memory: the ring of B stages (hi rows, then lo rows), then the ring of X/Y factor blocks
    auto stage_ptr = [&](int slot) { return smem + (size_t)slot * p.stage_bytes; };
    uint8_t* const xy_base = smem + (size_t)NS * p.stage_bytes;
    auto xy_ptr = [&](int slot) { return xy_base + (size_t)slot * (kXBlockBytes + kYBlockBytes); };
    uint8_t* const tail_base = xy_base + (size_t)kXyStages * (kXBlockBytes + kYBlockBytes);  // if bmax > 192

    if (tid == 0) {
        abort_flag = 0;
        for (int s = 0; s < NS; ++s) {
            trj_mbar_init(&full_b[s], 1);
            trj_mbar_init(&empty_b[s], 1);
        }
        for (int s = 0; s < kXyStages; ++s) {
            trj_mbar_init(&full_xy[s], 1);
            trj_mbar_init(&empty_xy[s], kBuildWarps);
        }
        for (int b = 0; b < k1MaxABufs; ++b) {
            trj_mbar_init(&full_a[b], kBuildWarps);
            trj_mbar_init(&empty_a[b], 1);
        }
        trj_mbar_init(&acc_full, 1);
        trj_mbar_init(&acc_empty, k1EpiWarps);
        trj_mbar_init(&mma_done, 1);
        trj_fence_mbar_init();
    }
    if (warp == k1MmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         trj_smem_addr(&tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (warp == k1TmaWarp) {
        if (lane == 0) {
            // ring position of the next stage (slot, phase) kept incrementally: no divisions per stage
            int slot = 0, issued = 0;
            unsigned phase = 0;
            for (int li = item0; li < item1 && !abort_flag; ++li) {
                const int it = p.cta_items[li];
                const TcTile T = p.tiles[it % p.ntiles];
                const TcChunk C = p.chunks[it / p.ntiles];
                const int nst = (C.slot1 - C.slot0) / kStageSlots;
                const unsigned bytes = (unsigned)(2 * T.ncols * 128);
                const int n64 = T.ncols / 64;  // B rows as 64-row boxes, then 16-row boxes
                for (int s = 0; s < nst; ++s) {
                    if (!timed_wait(&empty_b[slot], phase ^ 1, p.status)) {
                        abort_flag = 1;
                        break;
                    }
                    uint8_t* bh = stage_ptr(slot);
                    uint8_t* bl = bh + p.bmax * 128;
                    trj_mbar_arrive_expect_tx(&full_b[slot], bytes);
                    const int slot0 = C.slot0 + s * kStageSlots;
                    // rows of this stage's 32-slot block: contiguous 128-byte rows from row0
                    const int row0 = (slot0 / kStageSlots) * p.table_rows + T.brow;
                    int r = 0;
                    for (int b = 0; b < n64; ++b, r += 64) {
                        tma_load_2d(bh + r * 128, &map_hi64, 0, row0 + r, &full_b[slot]);
                        tma_load_2d(bl + r * 128, &map_lo64, 0, row0 + r, &full_b[slot]);
                    }
                    for (; r < T.ncols; r += 16) {
                        tma_load_2d(bh + r * 128, &map_hi, 0, row0 + r, &full_b[slot]);
                        tma_load_2d(bl + r * 128, &map_lo, 0, row0 + r, &full_b[slot]);
                    }
                    ++issued;
                    if (++slot == NS) {
                        slot = 0;
                        phase ^= 1;
                    }
                }
            }
            // the copies issued last land before the CTA may exit (they have, unless a wait gave up):
            // walk the ring back over the last min(issued, NS) stages
            for (int q = 0; q < NS && q < issued; ++q) {
                if (--slot < 0) {
                    slot = NS - 1;
                    phase ^= 1;
                }
                trj_mbar_wait(&full_b[slot], phase);
            }
        }
    } else if (warp == k1XyWarp) {
        if (lane == 0) {
            // X and Y factor blocks of every stage, released by the builders once they have read them
            int slot = 0, issued = 0;
            unsigned phase = 0;
            for (int li = item0; li < item1 && !abort_flag; ++li) {
                const int it = p.cta_items[li];
                const TcTile T = p.tiles[it % p.ntiles];
                const TcChunk C = p.chunks[it / p.ntiles];
                const int nst = (C.slot1 - C.slot0) / kStageSlots;
                const int bx = (T.nx0 - p.nx0min) / kTcTileNx, by = (T.ny0 - p.ny0min) / kTcTileNy;
                for (int s = 0; s < nst; ++s) {
                    if (!timed_wait(&empty_xy[slot], phase ^ 1, p.status)) {
                        abort_flag = 1;
                        break;
                    }
                    uint8_t* xf = xy_ptr(slot);
                    trj_mbar_arrive_expect_tx(&full_xy[slot], (unsigned)(kXBlockBytes + kYBlockBytes));
                    const int64_t stg = (C.slot0 + s * kStageSlots) / kStageSlots;
                    trj_bulk_g2s(xf, p.xtab + (stg * p.nxb + bx) * (kXBlockBytes / 16), kXBlockBytes, &full_xy[slot]);
                    trj_bulk_g2s(xf + kXBlockBytes, p.ytab + (stg * p.nyb + by) * (kYBlockBytes / 16), kYBlockBytes,
                                 &full_xy[slot]);
                    ++issued;
                    if (++slot == kXyStages) {
                        slot = 0;
                        phase ^= 1;
                    }
                }
            }
            for (int q = 0; q < kXyStages && q < issued; ++q) {
                if (--slot < 0) {
                    slot = kXyStages - 1;
                    phase ^= 1;
                }
                trj_mbar_wait(&full_xy[slot], phase);
            }
        }
    } else if (warp == k1MmaWarp) {
        if (lane == 0) {
            // B descriptor of stage slot 0; slot k sits k * stage_bytes further (the start-address
            // field holds addr >> 4 in 14 bits, which covers all of shared memory, so the offset adds
            // without carry).  A K-step of 16 bf16 (32 bytes) adds 2; the lo operand of B sits bmax
            // rows after the hi one.  A K-step of A in TMEM is 8 columns.
            const uint64_t b0desc = sw128_desc(trj_smem_addr(stage_ptr(0)));
            const uint64_t b_lo = (uint64_t)((p.bmax * 128) >> 4);
            const uint64_t b_step = (uint64_t)(p.stage_bytes >> 4);
            int slot = 0, fg = 0, ab = 0;
            unsigned phase = 0, aphase = 0;  // B ring phase; A ring (NA half-stage buffers) phase
            uint64_t bh = b0desc;            // B descriptor of the current slot
            for (int li = item0; li < item1 && !abort_flag; ++li) {
                const int it = p.cta_items[li];
                const TcTile T = p.tiles[it % p.ntiles];
                const TcChunk C = p.chunks[it / p.ntiles];
                const int nst = (C.slot1 - C.slot0) / kStageSlots;
                const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(T.ncols >> 3) << 17) |
                                       ((uint32_t)(128 >> 4) << 24);
                int rs = 0;  // stage within the current run
                for (int s = 0; s < nst; ++s) {
                    const bool first = rs == 0;
                    // the epilogue must have read the previous run out of the accumulator
                    if (first && fg >= 1 && !timed_wait(&acc_empty, (fg - 1) & 1, p.status)) {
                        abort_flag = 1;
                        break;
                    }
                    if (!timed_wait(&full_b[slot], phase, p.status)) {
                        abort_flag = 1;
                        break;
                    }
                    const uint64_t bl = bh + b_lo;
                    bool ok = true;
                    for (int hh = 0; hh < 2 && ok; ++hh) {
                        const int hb = ab;
                        if (!timed_wait(&full_a[hb], aphase, p.status)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t ah = tmem + p.a_col + (uint32_t)(32 * hb), al = ah + 16;
#pragma unroll
                        for (int k2 = 0; k2 < 2; ++k2) {
                            const int kk = 2 * hh + k2;
                            mma_ts(tmem, ah + 8 * k2, bh + 2 * kk, idesc, (first && kk == 0) ? 0u : 1u);
                            mma_ts(tmem, ah + 8 * k2, bl + 2 * kk, idesc, 1u);
                            mma_ts(tmem, al + 8 * k2, bh + 2 * kk, idesc, 1u);
                        }
                        mma_commit(&empty_a[hb]);
                        if (++ab == NA) {
                            ab = 0;
                            aphase ^= 1;
                        }
                    }
                    if (!ok) {
                        abort_flag = 1;
                        break;
                    }
                    mma_commit(&empty_b[slot]);
                    if (++rs == F || s == nst - 1) {
                        mma_commit(&acc_full);
                        ++fg;
                        rs = 0;
                    }
                    bh += b_step;
                    if (++slot == NS) {
                        slot = 0;
                        phase ^= 1;
                        bh = b0desc;
                    }
                }
            }
            // every MMA of this CTA has completed before TMEM is released
            mma_commit(&mma_done);
            trj_mbar_wait(&mma_done, 0);
        }
    } else if (warp >= k1EpiWarp0) {
        // ---- epilogue: each run of the accumulator is added (round to nearest) into an FP32 running
        //      sum; the item's last run writes sum + run to this CTA's FP32 block once.  Warp (quarter
        //      q4, group cg) owns the 8-column chunks cg, cg + 4, cg + 8, ... of TMEM lanes
        //      32 q4 .. 32 q4 + 31 (the tile's rows): the first k1RegChunks in registers, the one at
        //      columns >= k1TailCol in this warp's shared-memory tail. ----
        const int q4 = warp & 3;
        const int cg = (warp - k1EpiWarp0) >> 2;
        const int row = 32 * q4 + lane;
        // this warp's first column in TMEM (lane quarter in the high half); chunk i sits 32 i further
        const uint32_t ta = tmem + ((uint32_t)(32 * q4) << 16) + (uint32_t)(8 * cg);
        float* tail = reinterpret_cast<float*>(tail_base) + (warp - k1EpiWarp0) * 256 + lane;  // [8][32]
        float sum[k1RegChunks][8];
        int fg = 0;
        bool stop = false;
        for (int li = item0; li < item1 && !stop; ++li) {
            const int it = p.cta_items[li];
            const TcTile T = p.tiles[it % p.ntiles];
            const int chunk = it / p.ntiles;
            const TcChunk C = p.chunks[chunk];
            const int nst = (C.slot1 - C.slot0) / kStageSlots;
            const int nflush = (nst + F - 1) / F;
            const int lim = T.ncols - 8 * cg;  // chunk i is in the tile when 32 i < lim
            float* dst = p.part + (int64_t)chunk * p.acc_stride + T.acc_off + (int64_t)(8 * cg) * 128 + row;
            for (int f = 0; f < nflush; ++f, ++fg) {
                const bool ok = trj_mbar_wait(&acc_full, fg & 1);
                if (!__all_sync(0xffffffffu, ok)) {
                    if (lane == 0) trj_raise(p.status, TRJ_DEV_TIMEOUT);
                    abort_flag = 1;
                    stop = true;
                    break;
                }
                tc_fence_after();
                const bool last = f == nflush - 1;
#pragma unroll
                for (int i = 0; i < k1RegChunks; ++i) {
                    if (32 * i < lim) {  // warp-uniform
                        uint32_t a[8];
                        tmem_ld8_nowait(ta + (uint32_t)(32 * i), a);
                        tmem_wait_ld();
#pragma unroll
                        for (int k = 0; k < 8; ++k)
                            sum[i][k] = f > 0 ? __fadd_rn(__uint_as_float(a[k]), sum[i][k]) : __uint_as_float(a[k]);
                    }
                }
                if (k1TailCol < lim) {
                    uint32_t a[8];
                    tmem_ld8_nowait(ta + (uint32_t)k1TailCol, a);
                    tmem_wait_ld();
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        const float v = f > 0 ? __fadd_rn(__uint_as_float(a[k]), tail[32 * k]) : __uint_as_float(a[k]);
                        if (last) dst[(k1TailCol + k) * 128] = v;
                        else tail[32 * k] = v;
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) trj_mbar_arrive(&acc_empty);
                if (last) {
#pragma unroll
                    for (int i = 0; i < k1RegChunks; ++i) {
                        if (32 * i < lim) {
#pragma unroll
                            for (int k = 0; k < 8; ++k) dst[(32 * i + k) * 128] = sum[i][k];
                        }
                    }
                }
            }
        }
    } else {
        // ---- A builders (warps 0-7): warp w writes TMEM lanes 32*(w%4).. (A rows m) and, in each
        //      half-stage buffer, the K-columns of atoms [kHalfAtoms*(w/4), kHalfAtoms*(w/4 + 1)) ----
        const int q = warp & 3, g = warp >> 2;
        const int m = 32 * q + lane;
        const int nxl = m & 15, nyl = m >> 4;
        const uint32_t lanes = (uint32_t)(32 * q) << 16;
        int ab = 0, slot = 0;
        unsigned aphase = 0, phase = 0;  // A ring (NA half-stage buffers) in the MMA warp's order; X/Y ring
        bool stop = false;
        for (int li = item0; li < item1 && !stop; ++li) {
            const int it = p.cta_items[li];
            const TcChunk C = p.chunks[it / p.ntiles];
            const int nst = (C.slot1 - C.slot0) / kStageSlots;
            for (int s = 0; s < nst && !stop; ++s) {
                // the stage's X and Y factor blocks
                const bool ok = trj_mbar_wait(&full_xy[slot], phase);
                if (__any_sync(0xffffffffu, !ok || abort_flag)) {
                    if (lane == 0) trj_raise(p.status, TRJ_DEV_TIMEOUT);
                    abort_flag = 1;
                    stop = true;
                    break;
                }
                const float4* xf = reinterpret_cast<const float4*>(xy_ptr(slot));
                const float4* yf = xf + kXBlockBytes / 16;
                // Half-stage 0 is built and stored, half-stage 1 built while those stores drain; then
                // each half is released to the MMA warp once its own stores are complete.
                const int hb0 = ab;
                if (!__all_sync(0xffffffffu, trj_mbar_wait(&empty_a[hb0], aphase ^ 1))) {
                    if (lane == 0) trj_raise(p.status, TRJ_DEV_TIMEOUT);
                    abort_flag = 1;
                    stop = true;
                    break;
                }
                if (++ab == NA) {
                    ab = 0;
                    aphase ^= 1;
                }
                tc_fence_after();
                uint32_t hw[kHalfAtoms], lw[kHalfAtoms];
                build_row_tab(xf, yf, nxl, nyl, (kHalfAtoms * g) / 2, hw, lw);
                const uint32_t ta0 = tmem + lanes + p.a_col + (uint32_t)(32 * hb0 + kHalfAtoms * g);
                tmem_st_cols<kHalfAtoms>(ta0, hw);
                tmem_st_cols<kHalfAtoms>(ta0 + 16, lw);
                const int hb1 = ab;
                const bool ok1 = trj_mbar_wait(&empty_a[hb1], aphase ^ 1);
                if (++ab == NA) {
                    ab = 0;
                    aphase ^= 1;
                }
                uint32_t hw1[kHalfAtoms], lw1[kHalfAtoms];
                build_row_tab(xf, yf, nxl, nyl, (16 + kHalfAtoms * g) / 2, hw1, lw1);
                // every read of this stage's factor blocks is done: hand the buffer back
                __syncwarp();
                if (lane == 0) trj_mbar_arrive(&empty_xy[slot]);
                tmem_wait_st();  // half-stage 0's stores
                tc_fence_before();
                __syncwarp();
                if (lane == 0) trj_mbar_arrive(&full_a[hb0]);
                if (!__all_sync(0xffffffffu, ok1)) {
                    if (lane == 0) trj_raise(p.status, TRJ_DEV_TIMEOUT);
                    abort_flag = 1;
                    stop = true;
                    break;
                }
                tc_fence_after();
                const uint32_t ta1 = tmem + lanes + p.a_col + (uint32_t)(32 * hb1 + kHalfAtoms * g);
                tmem_st_cols<kHalfAtoms>(ta1, hw1);
                tmem_st_cols<kHalfAtoms>(ta1 + 16, lw1);
                tmem_wait_st();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) trj_mbar_arrive(&full_a[hb1]);
                if (++slot == kXyStages) {
                    slot = 0;
                    phase ^= 1;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == k1MmaWarp) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

// ---- CTA-pair (cta_group::2) form -------------------------------------------
// A cluster of two CTAs on a pair of SMs computes two tiles that share their B rows with one
// M = 256 tcgen05.mma per K-step: the leader (cluster rank 0) issues the MMAs; each CTA builds
// its own tile's A into its own TMEM and holds half of B's rows (N/2 each) in its own shared
// memory, so each SM reads half the B bytes of the one-CTA form from L2.  Loads of both CTAs
// complete on the leader's full_b barrier (TMA .cta_group::2 form, no multicast), the peer's
// producers and epilogue arrive on the leader's barriers through their cluster addresses, and
// the leader's commits arrive on both CTAs' barriers (multicast commit).

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// Address of the same shared-memory location in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(trj_smem_addr(p)), "r"(rank));
    return r;
}

__device__ __forceinline__ void remote_arrive(uint32_t cluster_bar) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_bar) : "memory");
}

// trj_mbar_wait with cluster-scope acquire (arrivals that come from the other CTA of the pair).
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar, unsigned parity) {
    const uint32_t addr = trj_smem_addr(bar);
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity), "r"(TRJ_SUSPEND_NS)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > TRJ_WAIT_CLOCKS) return false;
    }
}

__device__ __forceinline__ bool timed_wait_cluster(uint64_t* bar, unsigned parity, unsigned* status) {
    if (mbar_wait_cluster(bar, parity)) return true;
    trj_raise(status, TRJ_DEV_TIMEOUT);
    return false;
}

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// 2-D TMA load into this CTA's shared memory whose completion is counted on the leader's barrier.
__device__ __forceinline__ void tma_load_2d_pair(void* dst, const CUtensorMap* map, int c0, int c1,
                                                 uint32_t leader_bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
        "%3}], [%4];" ::"r"(trj_smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(leader_bar)
        : "memory");
}

__device__ __forceinline__ void mma_ts_pair(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(tmem_d),
        "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accum)
        : "memory");
}

// Arrive on the barrier at this offset in both CTAs of the pair once the leader's MMAs so far are done.
__device__ __forceinline__ void mma_commit_pair(uint64_t* bar) {
    const uint16_t mask = 3;
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            trj_smem_addr(bar)),
        "h"(mask)
        : "memory");
}

__global__ void __launch_bounds__(kTcThreads, 1)
    sq_tc2_kernel(const __grid_constant__ CUtensorMap map_hi, const __grid_constant__ CUtensorMap map_lo,
                  const __grid_constant__ CUtensorMap map_hi64, const __grid_constant__ CUtensorMap map_lo64,
                  Tc2Params p) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    // full_b, full_a, acc_empty are used in the leader only; the others in both CTAs
    __shared__ __align__(8) uint64_t full_b[kMaxStages], full_u[kMaxStages], empty_b[kMaxStages];
    __shared__ __align__(8) uint64_t full_a[kPairABufs], empty_a[kPairABufs], xy_full[2], xy_empty[2], acc_full,
        acc_empty, mma_done;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag_s;
    volatile int& abort_flag = abort_flag_s;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t rank = cluster_rank();
    const bool leader = rank == 0;
    const int cl = blockIdx.x >> 1;
    const int NS = p.nstages;
    const int F = p.flush_stages;
    const int item0 = p.cl_off[cl], item1 = p.cl_off[cl + 1];
    auto stage_ptr = [&](int slot) { return smem + (size_t)slot * p.stage_bytes; };
    auto xy_ptr = [&](int b) { return reinterpret_cast<float2*>(smem + (size_t)NS * p.stage_bytes + b * kXyBytes); };
    // FP32 running sum of this CTA's 128 accumulator rows: [16-column chunk][4 x 4 columns][row] float4
    float4* sums = reinterpret_cast<float4*>(smem + (size_t)NS * p.stage_bytes + 2 * kXyBytes);

    if (tid == 0) {
        abort_flag = 0;
        for (int s = 0; s < NS; ++s) {
            trj_mbar_init(&full_b[s], 1);
            trj_mbar_init(&full_u[s], 1);
            trj_mbar_init(&empty_b[s], 1);
        }
        for (int b = 0; b < kPairABufs; ++b) {
            trj_mbar_init(&full_a[b], 2 * kBuildWarps);
            trj_mbar_init(&empty_a[b], 1);
        }
        for (int b = 0; b < 2; ++b) {
            trj_mbar_init(&xy_full[b], kXyWarps);
            trj_mbar_init(&xy_empty[b], kBuildWarps);
        }
        trj_mbar_init(&acc_full, 1);
        trj_mbar_init(&acc_empty, 2 * kEpiWarps);
        trj_mbar_init(&mma_done, 1);
        trj_fence_mbar_init();
    }
    if (warp == kMmaWarp) {  // the same warp of both CTAs allocates the pair's TMEM
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         trj_smem_addr(&tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    cluster_sync_all();  // barrier inits and TMEM of both CTAs visible to both
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (warp == kTmaWarp) {
        if (lane == 0) {
            int slot = 0, issued = 0;
            unsigned phase = 0;
            for (int li = item0; li < item1 && !abort_flag; ++li) {
                const int it = p.cl_items[li];
                const TcPairDev P = p.pairs[it % p.npairs];
                const TcChunk C = p.chunks[it / p.npairs];
                const int nst = (C.slot1 - C.slot0) / kStageSlots;
                const int half = P.ncols / 2;                 // B rows of this CTA
                const int row0 = P.brow + (int)rank * half;
                const int n64 = half / 64;
                for (int s = 0; s < nst; ++s) {
                    if (!timed_wait(&empty_b[slot], phase ^ 1, p.status)) {
                        abort_flag = 1;
                        break;
                    }
                    uint8_t* bh = stage_ptr(slot);
                    uint8_t* bl = bh + p.bhalf * 128;
                    uint8_t* ux = bl + p.bhalf * 128;
                    const uint32_t lead_full = cluster_addr(&full_b[slot], 0);
                    if (leader) trj_mbar_arrive_expect_tx(&full_b[slot], (unsigned)(P.ncols * 256));
                    trj_mbar_arrive_expect_tx(&full_u[slot], (unsigned)kUxyBytes);
                    const int slot0 = C.slot0 + s * kStageSlots;
                    const int rowb = (slot0 / kStageSlots) * p.table_rows + row0;  // this stage's block
                    int r = 0;
                    for (int b = 0; b < n64; ++b, r += 64) {
                        tma_load_2d_pair(bh + r * 128, &map_hi64, 0, rowb + r, lead_full);
                        tma_load_2d_pair(bl + r * 128, &map_lo64, 0, rowb + r, lead_full);
                    }
                    for (; r < half; r += 16) {
                        tma_load_2d_pair(bh + r * 128, &map_hi, 0, rowb + r, lead_full);
                        tma_load_2d_pair(bl + r * 128, &map_lo, 0, rowb + r, lead_full);
                    }
                    trj_bulk_g2s(ux, p.uxy + slot0, kUxyBytes, &full_u[slot]);
                    ++issued;
                    if (++slot == NS) {
                        slot = 0;
                        phase ^= 1;
                    }
                }
            }
            // copies issued last land before the CTA may exit (the leader's full_b counts both CTAs')
            for (int q = 0; q < NS && q < issued; ++q) {
                if (--slot < 0) {
                    slot = NS - 1;
                    phase ^= 1;
                }
                trj_mbar_wait(&full_u[slot], phase);
                if (leader) mbar_wait_cluster(&full_b[slot], phase);
            }
        }
    } else if (warp == kMmaWarp) {
        if (lane == 0 && leader) {
            const uint64_t b0desc = sw128_desc(trj_smem_addr(stage_ptr(0)));
            const uint64_t b_lo = (uint64_t)((p.bhalf * 128) >> 4);
            const uint64_t b_step = (uint64_t)(p.stage_bytes >> 4);
            int slot = 0, fg = 0, ab = 0;
            unsigned phase = 0, aphase = 0;
            uint64_t bh = b0desc;
            for (int li = item0; li < item1 && !abort_flag; ++li) {
                const int it = p.cl_items[li];
                const TcPairDev P = p.pairs[it % p.npairs];
                const TcChunk C = p.chunks[it / p.npairs];
                const int nst = (C.slot1 - C.slot0) / kStageSlots;
                const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(P.ncols >> 3) << 17) |
                                       ((uint32_t)(256 >> 4) << 24);
                int rs = 0;
                for (int s = 0; s < nst; ++s) {
                    const bool first = rs == 0;
                    if (first && fg >= 1 && !timed_wait_cluster(&acc_empty, (fg - 1) & 1, p.status)) {
                        abort_flag = 1;
                        break;
                    }
                    if (!timed_wait_cluster(&full_b[slot], phase, p.status)) {
                        abort_flag = 1;
                        break;
                    }
                    const uint64_t bl = bh + b_lo;
                    if (!timed_wait_cluster(&full_a[ab], aphase, p.status)) {
                        abort_flag = 1;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t ah = tmem + kPairACol + (uint32_t)(64 * ab), al = ah + 32;
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        mma_ts_pair(tmem, ah + 8 * kk, bh + 2 * kk, idesc, (first && kk == 0) ? 0u : 1u);
                        mma_ts_pair(tmem, ah + 8 * kk, bl + 2 * kk, idesc, 1u);
                        mma_ts_pair(tmem, al + 8 * kk, bh + 2 * kk, idesc, 1u);
                    }
                    mma_commit_pair(&empty_a[ab]);
                    mma_commit_pair(&empty_b[slot]);
                    if (++rs == F || s == nst - 1) {
                        mma_commit_pair(&acc_full);
                        ++fg;
                        rs = 0;
                    }
                    if (++ab == kPairABufs) {
                        ab = 0;
                        aphase ^= 1;
                    }
                    bh += b_step;
                    if (++slot == NS) {
                        slot = 0;
                        phase ^= 1;
                        bh = b0desc;
                    }
                }
            }
            mma_commit_pair(&mma_done);  // every MMA of the pair has completed -> both CTAs
        }
        if (lane == 0) trj_mbar_wait(&mma_done, 0);
    } else if (warp >= kEpiWarp0) {
        const int q4 = warp & 3;
        const int c0 = 16 * ((warp - kEpiWarp0) >> 2);
        const int row = 32 * q4 + lane;
        const uint32_t lanes = (uint32_t)(32 * q4) << 16;
        const uint32_t lead_acc_empty = cluster_addr(&acc_empty, 0);
        int fg = 0;
        bool stop = false;
        for (int li = item0; li < item1 && !stop; ++li) {
            const int it = p.cl_items[li];
            const TcPairDev P = p.pairs[it % p.npairs];
            const int chunk = it / p.npairs;
            const TcChunk C = p.chunks[chunk];
            const int nst = (C.slot1 - C.slot0) / kStageSlots;
            const int nflush = (nst + F - 1) / F;
            const int tile = P.tile[rank];
            const int coff = P.coff[rank];
            int own = 0;
            float* dst = nullptr;
            if (tile >= 0) {
                const TcTile T = p.tiles[tile];
                own = T.ncols;
                dst = p.part + (int64_t)chunk * p.acc_stride + T.acc_off + row;
            }
            for (int f = 0; f < nflush; ++f, ++fg) {
                const bool ok = trj_mbar_wait(&acc_full, fg & 1);
                if (!__all_sync(0xffffffffu, ok)) {
                    if (lane == 0) trj_raise(p.status, TRJ_DEV_TIMEOUT);
                    abort_flag = 1;
                    stop = true;
                    break;
                }
                tc_fence_after();
                const bool last = f == nflush - 1;
                const uint32_t ta = tmem + lanes;
                for (int c = c0; c < P.ncols; c += 32) {
                    uint32_t a0[16];
                    tmem_ld16_nowait(ta + (uint32_t)c, a0);
                    tmem_wait_ld();
                    float4* sp = sums + (size_t)(c >> 4) * 4 * 128 + row;  // this row's 4 float4 of the chunk
#pragma unroll
                    for (int k4 = 0; k4 < 4; ++k4) {
                        float4 v = make_float4(__uint_as_float(a0[4 * k4]), __uint_as_float(a0[4 * k4 + 1]),
                                               __uint_as_float(a0[4 * k4 + 2]), __uint_as_float(a0[4 * k4 + 3]));
                        if (f > 0) {
                            const float4 o = sp[k4 * 128];
                            v.x = __fadd_rn(v.x, o.x), v.y = __fadd_rn(v.y, o.y);
                            v.z = __fadd_rn(v.z, o.z), v.w = __fadd_rn(v.w, o.w);
                        }
                        if (last) {
                            if (dst) {
                                const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                                for (int e = 0; e < 4; ++e) {
                                    const int oc = c + 4 * k4 + e - coff;  // own column
                                    if (oc >= 0 && oc < own) dst[(int64_t)oc * 128] = vv[e];
                                }
                            }
                        } else {
                            sp[k4 * 128] = v;
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    if (leader) trj_mbar_arrive(&acc_empty);
                    else remote_arrive(lead_acc_empty);
                }
            }
        }
    } else if (warp >= kXyWarp0) {
        const int xt = tid - kXyWarp0 * 32;
        int sg = 0, slot = 0;
        unsigned phase = 0;
        bool stop = false;
        for (int li = item0; li < item1 && !stop; ++li) {
            const int it = p.cl_items[li];
            const TcPairDev P = p.pairs[it % p.npairs];
            const TcChunk C = p.chunks[it / p.npairs];
            const int nst = (C.slot1 - C.slot0) / kStageSlots;
            const int nx0 = P.nx0[rank], ny0 = P.ny0[rank];
            for (int s = 0; s < nst; ++s, ++sg) {
                const int xb = sg & 1;
                bool ok = trj_mbar_wait(&full_u[slot], phase);
                ok = ok && trj_mbar_wait(&xy_empty[xb], ((sg >> 1) & 1) ^ 1);
                if (__any_sync(0xffffffffu, !ok || abort_flag)) {
                    if (lane == 0) trj_raise(p.status, TRJ_DEV_TIMEOUT);
                    abort_flag = 1;
                    stop = true;
                    break;
                }
                const uint2* u = reinterpret_cast<const uint2*>(stage_ptr(slot) + 2 * p.bhalf * 128);
                fill_xy(xy_ptr(xb), u, nx0, ny0, xt, kXyWarps * 32);
                __syncwarp();
                if (lane == 0) trj_mbar_arrive(&xy_full[xb]);
                if (++slot == NS) {
                    slot = 0;
                    phase ^= 1;
                }
            }
        }
    } else {
        // ---- A builders: warp w writes TMEM lanes 32*(w%4).. and the K-columns of atoms
        //      [2*kHalfAtoms*(w/4), 2*kHalfAtoms*(w/4 + 1)) of the stage's A buffer, arriving on the
        //      leader's full_a ----
        const int q = warp & 3, g = warp >> 2;
        const int m = 32 * q + lane;
        const int nxl = m & 15, nyl = m >> 4;
        const uint32_t lanes = (uint32_t)(32 * q) << 16;
        int sg = 0, ab = 0;
        unsigned aphase = 0;
        bool stop = false;
        for (int li = item0; li < item1 && !stop; ++li) {
            const int it = p.cl_items[li];
            const TcChunk C = p.chunks[it / p.npairs];
            const int nst = (C.slot1 - C.slot0) / kStageSlots;
            for (int s = 0; s < nst && !stop; ++s, ++sg) {
                const int xb = sg & 1;
                bool ok = trj_mbar_wait(&xy_full[xb], (sg >> 1) & 1);
                ok = ok && trj_mbar_wait(&empty_a[ab], aphase ^ 1);
                if (__any_sync(0xffffffffu, !ok || abort_flag)) {
                    if (lane == 0) trj_raise(p.status, TRJ_DEV_TIMEOUT);
                    abort_flag = 1;
                    stop = true;
                    break;
                }
                tc_fence_after();
                const float2* xs = xy_ptr(xb);
                const uint32_t ta = tmem + lanes + kPairACol + (uint32_t)(64 * ab + 2 * kHalfAtoms * g);
#pragma unroll
                for (int h8 = 0; h8 < 2 * kHalfAtoms / 8; ++h8) {
                    uint32_t hw[8], lw[8];
                    build_row<8>(xs, nxl, nyl, 2 * kHalfAtoms * g + 8 * h8, hw, lw);
                    tmem_st8(ta + 8 * h8, hw);
                    tmem_st8(ta + 32 + 8 * h8, lw);
                }
                tmem_wait_st();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    trj_mbar_arrive(&xy_empty[xb]);
                    if (leader) trj_mbar_arrive(&full_a[ab]);
                    else remote_arrive(cluster_addr(&full_a[ab], 0));
                }
                if (++ab == kPairABufs) {
                    ab = 0;
                    aphase ^= 1;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync_all();  // neither CTA leaves while the other may still reach its barriers or TMEM
    if (warp == kMmaWarp) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

// tc_out[tile][a][col][row] = sum over species a's chunks (fixed order) of the FP64 blocks.
// Grid (element blocks, tile, species): one thread per output element.
__global__ void tc_reduce_kernel(const float* __restrict__ part, int64_t acc_stride, const TcTile* __restrict__ tiles,
                                 const SqTile* __restrict__ stiles, const int32_t* __restrict__ chunk_begin, int nsp,
                                 double* __restrict__ out) {
    const int t = blockIdx.y, a = blockIdx.z;
    const TcTile T = tiles[t];
    const int64_t n = (int64_t)T.ncols * 128;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int k0 = chunk_begin[a], k1 = chunk_begin[a + 1];
    const float* src = part + T.acc_off + e;
    double s = 0.0;
    for (int k = k0; k < k1; ++k) s += (double)__ldcs(src + (int64_t)k * acc_stride);
    out[stiles[t].out_off + (int64_t)a * n + e] = s;
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

// 2-D map over a row-major [rows][inner] array; inner extent and box inner in elements.
int encode_map(trj_ctx* ctx, CUtensorMap* map, void* base, CUtensorMapDataType dt, int esize, int64_t inner,
               int64_t rows, int box_inner, int box_rows, CUtensorMapSwizzle sw) {
    EncodeTiledFn enc = get_encode();
    if (!enc) return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)inner * esize};
    cuuint32_t box[2] = {(cuuint32_t)box_inner, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, dt, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return trj_fail(ctx, TRJ_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return TRJ_OK;
}

}  // namespace

void trj_sq_tc_release(trj_sq_plan* plan) {
    TcState* st = reinterpret_cast<TcState*>(plan->tc_state);
    if (!st) return;
    void* ptrs[] = {st->sched_dev, st->tiles_dev, st->chunks_dev, st->pad_off_dev, st->chunk_begin_dev,
                    st->tab_hi,    st->tab_lo,    st->uxy,        st->part,           st->pairs_dev,
                    st->sched2_dev, st->xtab,     st->ytab};
    for (void* q : ptrs) trj_dev_free(plan->ctx, q);
    delete st;
    plan->tc_state = nullptr;
}

// CTA-pair form: pairs of tiles sharing their B rows, the per-cluster schedule and the launch
// shape.  Leaves pairs_ok = 0 (the one-CTA form runs) when the device cannot keep clusters of two
// resident with this shared-memory size.
static int prepare_pairs(trj_sq_plan* plan, TcState* st, const std::vector<TcTile>& tt) {
    trj_ctx* ctx = plan->ctx;
    const int ntiles = (int)tt.size();
    const int nz_min = st->nz_min;
    // tiles by descending span, then origin, so that neighbours have equal or nested nz ranges
    std::vector<int> ord(ntiles);
    for (int i = 0; i < ntiles; ++i) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
        if (tt[a].ncols != tt[b].ncols) return tt[a].ncols > tt[b].ncols;
        return plan->tiles[a].nz0 < plan->tiles[b].nz0;
    });
    std::vector<TcPairDev> pairs;
    for (size_t k = 0; k < ord.size();) {
        const int a = ord[k];
        const int za0 = plan->tiles[a].nz0, za1 = za0 + tt[a].ncols / 2 - 1;
        int b = k + 1 < ord.size() ? ord[k + 1] : -1;
        int z0 = za0, z1 = za1;
        if (b >= 0) {
            const int zb0 = plan->tiles[b].nz0, zb1 = zb0 + tt[b].ncols / 2 - 1;
            const int u0 = std::min(za0, zb0), u1 = std::max(za1, zb1);
            if (2 * (u1 - u0 + 1) <= kMaxTileCols) {
                z0 = u0;
                z1 = u1;
            } else {
                b = -1;
            }
        }
        TcPairDev P;
        P.tile[0] = a;
        P.tile[1] = b;
        P.ncols = (2 * (z1 - z0 + 1) + 31) / 32 * 32;
        P.brow = 2 * (z0 - nz_min);
        P.coff[0] = 2 * (za0 - z0);
        P.coff[1] = b >= 0 ? 2 * (plan->tiles[b].nz0 - z0) : 0;
        P.nx0[0] = tt[a].nx0;
        P.ny0[0] = tt[a].ny0;
        P.nx0[1] = b >= 0 ? tt[b].nx0 : tt[a].nx0;
        P.ny0[1] = b >= 0 ? tt[b].ny0 : tt[a].ny0;
        if (P.ncols > kMaxTileCols) return TRJ_OK;  // cannot happen: spans are <= kMaxTileCols / 2
        pairs.push_back(P);
        k += b >= 0 ? 2 : 1;
    }
    st->npairs = (int)pairs.size();
    int bmax2 = 0;
    for (const TcPairDev& P : pairs) bmax2 = std::max(bmax2, P.ncols);
    st->bhalf = bmax2 / 2;
    st->stage_bytes2 = (2 * st->bhalf * 128 + kUxyBytes + 1023) / 1024 * 1024;
    const int sum_bytes = bmax2 * 128 * 4;  // FP32 running sum of 128 rows x N
    const int avail = (int)ctx->smem_optin - 2048 - 2 * kXyBytes - sum_bytes;
    st->nstages2 = std::min(kMaxStages, avail / st->stage_bytes2);
    if (st->nstages2 < 2) return TRJ_OK;
    st->smem_bytes2 = st->nstages2 * st->stage_bytes2 + 2 * kXyBytes + sum_bytes + 1024;
    // resident clusters of two with this shared-memory size
    if (cudaFuncSetAttribute(sq_tc2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, st->smem_bytes2) !=
        cudaSuccess) {
        cudaGetLastError();
        return TRJ_OK;
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)(ctx->sm_count & ~1));
    cfg.blockDim = dim3(kTcThreads);
    cfg.dynamicSmemBytes = (size_t)st->smem_bytes2;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int ncl = 0;
    if (cudaOccupancyMaxActiveClusters(&ncl, (void*)sq_tc2_kernel, &cfg) != cudaSuccess || ncl < 1) {
        cudaGetLastError();
        return TRJ_OK;
    }
    const int64_t nchunks = (int64_t)st->chunks.size();
    const int64_t nitems = (int64_t)st->npairs * nchunks;
    ncl = (int)std::min<int64_t>(ncl, nitems);
    st->grid2 = 2 * ncl;
    // windowed longest-first schedule over clusters (as for the one-CTA form)
    std::vector<std::vector<int32_t>> lists(ncl);
    std::vector<std::pair<double, int>> heap;
    for (int b = 0; b < ncl; ++b) heap.push_back({0.0, b});
    auto cmp = [](const std::pair<double, int>& a, const std::pair<double, int>& b) { return a > b; };
    std::make_heap(heap.begin(), heap.end(), cmp);
    std::vector<std::pair<double, int32_t>> win;
    for (int64_t w0 = 0; w0 < nitems; w0 += ncl) {
        win.clear();
        for (int64_t it = w0; it < std::min<int64_t>(nitems, w0 + ncl); ++it) {
            const TcChunk& C = st->chunks[it / st->npairs];
            const double stages = (double)(C.slot1 - C.slot0) / kStageSlots;
            win.push_back({stages * (pairs[it % st->npairs].ncols + 24.0), (int32_t)it});
        }
        std::stable_sort(win.begin(), win.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
        for (const auto& it : win) {
            std::pop_heap(heap.begin(), heap.end(), cmp);
            heap.back().first += it.first;
            lists[heap.back().second].push_back(it.second);
            std::push_heap(heap.begin(), heap.end(), cmp);
        }
    }
    std::vector<int32_t> sched(ncl + 1, 0);
    for (int b = 0; b < ncl; ++b) sched[b + 1] = sched[b] + (int32_t)lists[b].size();
    for (int b = 0; b < ncl; ++b) sched.insert(sched.end(), lists[b].begin(), lists[b].end());
    if (trj_dev_alloc(ctx, (void**)&st->pairs_dev, sizeof(TcPairDev) * pairs.size()) != cudaSuccess ||
        trj_dev_alloc(ctx, (void**)&st->sched2_dev, sizeof(int32_t) * sched.size()) != cudaSuccess)
        return trj_fail(ctx, TRJ_ERR_NOMEM, "tensor path: pair schedule");
    cudaMemcpy(st->pairs_dev, pairs.data(), sizeof(TcPairDev) * pairs.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(st->sched2_dev, sched.data(), sizeof(int32_t) * sched.size(), cudaMemcpyHostToDevice);
    st->pairs_ok = 1;
    return TRJ_OK;
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
    // Z-table extent and tile widths
    int nz_min = plan->tiles[0].nz0, nz_max = nz_min;
    for (const SqTile& t : plan->tiles) {
        nz_min = std::min(nz_min, t.nz0);
        nz_max = std::max(nz_max, t.nz0 + t.ncols / 2 - 1);
        st->bmax = std::max(st->bmax, t.ncols);
    }
    if (st->bmax > kMaxTileCols)
        return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "tensor path: tile of %d columns > %d", st->bmax, kMaxTileCols);
    st->nz_min = nz_min;
    st->table_rows = 2 * (nz_max - nz_min + 1);
    // A ring from the first multiple of 32 columns after the accumulator
    st->a_col = (st->bmax + 31) / 32 * 32;
    st->nabuf = std::min(k1MaxABufs, (int)(kTmemCols - st->a_col) / 32);  // 9 for every bmax <= 224
    const int ntiles = (int)plan->tiles.size();
    std::vector<TcTile> tt(ntiles);
    int64_t acc = 0;
    for (int i = 0; i < ntiles; ++i) {
        const SqTile& s = plan->tiles[i];
        tt[i] = TcTile{s.nx0, s.ny0, s.ncols, 2 * (s.nz0 - nz_min), acc};
        acc += (int64_t)s.ncols * 128;
    }
    st->acc_stride = acc;
    // chunks: each species' slots split into runs of about kChunkAtoms atoms, and into at least as
    // many chunks as it takes for tiles x chunks to cover the GPU a few times
    const int64_t target_chunks = std::max<int64_t>(nsp, (6 * ctx->sm_count + ntiles - 1) / ntiles);
    const int64_t total_real = std::max<int64_t>(1, plan->n_total);
    st->chunk_of_species_begin.assign(nsp + 1, 0);
    for (int a = 0; a < nsp; ++a) {
        st->chunk_of_species_begin[a] = (int)st->chunks.size();
        const int64_t slots = st->pad_off[a + 1] - st->pad_off[a];
        const int64_t stages = slots / kStageSlots;
        if (stages == 0) continue;
        int64_t k = std::max<int64_t>(1, (target_chunks * plan->species_counts[a] + total_real - 1) / total_real);
        k = std::max<int64_t>(k, (slots + kChunkAtoms - 1) / kChunkAtoms);
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
    // shared memory: a ring of B stages (hi rows, then lo rows; 256 * bmax bytes, a multiple of 4096,
    // so every stage starts on the 1024-byte boundary of the 128-byte swizzle), then the ring of
    // kXyStages X/Y factor-block stages
    st->stage_bytes = 2 * st->bmax * 128;
    // kXyStages X/Y factor-block stages, and for tiles wider than k1TailCol columns the epilogue's
    // shared-memory tail of the running sum
    const int xy_bytes = kXyStages * (kXBlockBytes + kYBlockBytes) + (st->bmax > k1TailCol ? k1TailBytes : 0);
    const int avail = (int)ctx->smem_optin - 2048 - xy_bytes;
    st->nstages = std::min(kMaxStages, avail / st->stage_bytes);
    if (st->nstages < 2) return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "tensor path: tile too wide for shared memory");
    st->smem_bytes = st->nstages * st->stage_bytes + xy_bytes + 1024;
    // X/Y factor blocks: every 16-nx (8-ny) block a tile starts at
    int nxmax = tt[0].nx0, nymax = tt[0].ny0;
    st->nx0min = tt[0].nx0;
    st->ny0min = tt[0].ny0;
    for (const TcTile& t : tt) {
        st->nx0min = std::min(st->nx0min, t.nx0);
        st->ny0min = std::min(st->ny0min, t.ny0);
        nxmax = std::max(nxmax, t.nx0);
        nymax = std::max(nymax, t.ny0);
    }
    st->nxb = (nxmax - st->nx0min) / kTcTileNx + 1;
    st->nyb = (nymax - st->ny0min) / kTcTileNy + 1;
    const int64_t nitems = (int64_t)ntiles * (int64_t)st->chunks.size();
    st->grid = (int)std::min<int64_t>(nitems, ctx->sm_count);
    // Schedule: the items in chunk-major order are cut into windows of `grid` items; within a window
    // each item (costed by (columns + A-build work) x stages, longest first) goes to the least-loaded
    // CTA.  Every CTA walks its items window by window, so at any time the CTAs stream the Z-table
    // rows of the same few chunks and the L2 serves each chunk to every tile.
    std::vector<int32_t> sched;
    {
        std::vector<std::vector<int32_t>> lists(st->grid);
        std::vector<std::pair<double, int>> heap;  // (load, cta), min-heap
        for (int b = 0; b < st->grid; ++b) heap.push_back({0.0, b});
        auto cmp = [](const std::pair<double, int>& a, const std::pair<double, int>& b) { return a > b; };
        std::make_heap(heap.begin(), heap.end(), cmp);
        std::vector<std::pair<double, int32_t>> win;
        for (int64_t w0 = 0; w0 < nitems; w0 += st->grid) {
            win.clear();
            for (int64_t it = w0; it < std::min<int64_t>(nitems, w0 + st->grid); ++it) {
                const TcChunk& C = st->chunks[it / ntiles];
                const double stages = (double)(C.slot1 - C.slot0) / kStageSlots;
                win.push_back({stages * (tt[it % ntiles].ncols + 24.0), (int32_t)it});
            }
            std::stable_sort(win.begin(), win.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
            for (const auto& it : win) {
                std::pop_heap(heap.begin(), heap.end(), cmp);
                heap.back().first += it.first;
                lists[heap.back().second].push_back(it.second);
                std::push_heap(heap.begin(), heap.end(), cmp);
            }
        }
        sched.assign(st->grid + 1, 0);
        for (int b = 0; b < st->grid; ++b) sched[b + 1] = sched[b] + (int32_t)lists[b].size();
        for (int b = 0; b < st->grid; ++b) sched.insert(sched.end(), lists[b].begin(), lists[b].end());
    }

    const int64_t kdim = 2 * st->total_slots;
    size_t tab_bytes = (size_t)st->table_rows * (size_t)kdim * sizeof(__nv_bfloat16);
    size_t uxy_bytes = sizeof(uint2) * (size_t)st->total_slots;
    const int64_t nstage_tot = st->total_slots / kStageSlots;
    const size_t xtab_bytes = (size_t)nstage_tot * st->nxb * kXBlockBytes;
    const size_t ytab_bytes = (size_t)nstage_tot * st->nyb * kYBlockBytes;
    size_t part_bytes = sizeof(float) * (size_t)st->acc_stride * st->chunks.size();
    std::vector<int32_t> cb(st->chunk_of_species_begin.begin(), st->chunk_of_species_begin.end());
    if (trj_dev_alloc(ctx, (void**)&st->tab_hi, tab_bytes) != cudaSuccess ||
        trj_dev_alloc(ctx, (void**)&st->tab_lo, tab_bytes) != cudaSuccess ||
        trj_dev_alloc(ctx, (void**)&st->uxy, uxy_bytes) != cudaSuccess ||
        trj_dev_alloc(ctx, (void**)&st->xtab, xtab_bytes) != cudaSuccess ||
        trj_dev_alloc(ctx, (void**)&st->ytab, ytab_bytes) != cudaSuccess ||
        trj_dev_alloc(ctx, (void**)&st->part, part_bytes) != cudaSuccess ||
        trj_dev_alloc(ctx, (void**)&st->tiles_dev, sizeof(TcTile) * tt.size()) != cudaSuccess ||
        trj_dev_alloc(ctx, (void**)&st->chunks_dev, sizeof(TcChunk) * st->chunks.size()) != cudaSuccess ||
        trj_dev_alloc(ctx, (void**)&st->pad_off_dev, sizeof(int64_t) * (2 * nsp + 1)) != cudaSuccess ||
        trj_dev_alloc(ctx, (void**)&st->chunk_begin_dev, sizeof(int32_t) * (nsp + 1)) != cudaSuccess ||
        trj_dev_alloc(ctx, (void**)&st->sched_dev, sizeof(int32_t) * sched.size()) != cudaSuccess)
        return trj_fail(ctx, TRJ_ERR_NOMEM, "tensor path: %zu bytes of tables",
                        2 * tab_bytes + uxy_bytes + xtab_bytes + ytab_bytes + part_bytes);
    cudaMemcpy(st->tiles_dev, tt.data(), sizeof(TcTile) * tt.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(st->chunks_dev, st->chunks.data(), sizeof(TcChunk) * st->chunks.size(), cudaMemcpyHostToDevice);
    // pad offsets, then the per-species slot -> atom multipliers
    std::vector<int64_t> pad_mul(st->pad_off.begin(), st->pad_off.end());
    for (int a = 0; a < nsp; ++a) {
        const int64_t na = plan->species_counts[a];
        int64_t m = na > 1 ? std::max<int64_t>(1, (int64_t)(0.6180339887498949 * (double)na + 0.5)) % na : 1;
        auto gcd = [](int64_t x, int64_t y) {
            while (y) {
                int64_t t = x % y;
                x = y;
                y = t;
            }
            return x;
        };
        while (na > 1 && (m == 0 || gcd(m, na) != 1)) m = (m + 1) % na;
        pad_mul.push_back(m);
    }
    cudaMemcpy(st->pad_off_dev, pad_mul.data(), sizeof(int64_t) * (2 * nsp + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(st->chunk_begin_dev, cb.data(), sizeof(int32_t) * (nsp + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(st->sched_dev, sched.data(), sizeof(int32_t) * sched.size(), cudaMemcpyHostToDevice);
    plan->scratch_bytes += (int64_t)(2 * tab_bytes + uxy_bytes + xtab_bytes + ytab_bytes + part_bytes);
    // Blocked table: [total_slots / 32][table_rows][64 bf16] as a 2-D map of 128-byte rows.
    const int64_t brows = (st->total_slots / kStageSlots) * (int64_t)st->table_rows;
    int rc = encode_map(ctx, &st->map_hi, st->tab_hi, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, 64, brows, 64, 16,
                        CU_TENSOR_MAP_SWIZZLE_128B);
    if (rc == TRJ_OK)
        rc = encode_map(ctx, &st->map_lo, st->tab_lo, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, 64, brows, 64, 16,
                        CU_TENSOR_MAP_SWIZZLE_128B);
    if (rc == TRJ_OK)
        rc = encode_map(ctx, &st->map_hi64, st->tab_hi, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, 64, brows, 64, 64,
                        CU_TENSOR_MAP_SWIZZLE_128B);
    if (rc == TRJ_OK)
        rc = encode_map(ctx, &st->map_lo64, st->tab_lo, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, 64, brows, 64, 64,
                        CU_TENSOR_MAP_SWIZZLE_128B);
    if (rc != TRJ_OK) return rc;
    TRJ_CUDA_TRY(ctx, cudaFuncSetAttribute(sq_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           st->smem_bytes));
    return prepare_pairs(plan, st, tt);
}

int trj_sq_tc_run(trj_sq_plan* plan, const float box[3], cudaStream_t s) {
    (void)box;
    trj_ctx* ctx = plan->ctx;
    TcState* st = reinterpret_cast<TcState*>(plan->tc_state);
    if (!st || !st->tab_hi)
        return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "tensor-core S(Q) path was not prepared for this plan");
    const int nz_count = st->table_rows / 2;
    // Four row groups per slot: each thread walks a quarter of the nz rows, so the slot -> atom
    // mapping (a 64-bit modulo) and the phase load are done 4 times per slot, not once per row group
    // of 32.
    dim3 zg((unsigned)((st->total_slots + 255) / 256), (unsigned)std::min(nz_count, 4));
    tc_ztable_kernel<<<zg, 256, 0, s>>>(plan->phase_dev, plan->species_off_dev, st->pad_off_dev, plan->nsp,
                                        st->total_slots, st->nz_min, nz_count, (int64_t)st->table_rows, st->tab_hi,
                                        st->tab_lo, st->uxy,
                                        plan->qsp >= 0 ? plan->n_atoms : INT64_MAX);
    const bool pair_form = st->pairs_ok && st->use_pairs;
    if (!pair_form) {  // the one-CTA form reads its X/Y factors from per-frame blocks
        const int64_t nstage_tot = st->total_slots / kStageSlots;
        const int64_t nent = nstage_tot * (st->nxb * (kStageSlots / 2) * kTcTileNx + st->nyb * (kStageSlots / 2) * kTcTileNy);
        tc_xytable_kernel<<<(unsigned)((nent + 255) / 256), 256, 0, s>>>(st->uxy, nstage_tot, st->nxb, st->nx0min,
                                                                         st->nyb, st->ny0min, st->xtab, st->ytab);
        ctx->launches += 1;
    }
    TcParams P;
    P.tiles = st->tiles_dev;
    P.chunks = st->chunks_dev;
    P.cta_off = st->sched_dev;
    P.cta_items = st->sched_dev + st->grid + 1;
    P.uxy = st->uxy;
    P.part = st->part;
    P.acc_stride = st->acc_stride;
    P.ntiles = (int)plan->tiles.size();
    P.nchunks = (int)st->chunks.size();
    P.nstages = st->nstages;
    P.flush_stages = st->flush_stages;
    P.stage_bytes = st->stage_bytes;
    P.bmax = st->bmax;
    P.table_rows = st->table_rows;
    P.a_col = (uint32_t)st->a_col;
    P.nabuf = st->nabuf;
    P.xtab = st->xtab;
    P.ytab = st->ytab;
    P.nxb = st->nxb;
    P.nyb = st->nyb;
    P.nx0min = st->nx0min;
    P.ny0min = st->ny0min;
    P.status = ctx->status_dev;
    // The attribute is per kernel, shared by all plans: set this plan's size right before its launch.
    TRJ_CUDA_TRY(ctx, cudaFuncSetAttribute(sq_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           st->smem_bytes));
    if (pair_form) {
        Tc2Params Q;
        Q.tiles = st->tiles_dev;
        Q.pairs = st->pairs_dev;
        Q.chunks = st->chunks_dev;
        Q.cl_off = st->sched2_dev;
        Q.cl_items = st->sched2_dev + st->grid2 / 2 + 1;
        Q.uxy = st->uxy;
        Q.part = st->part;
        Q.acc_stride = st->acc_stride;
        Q.npairs = st->npairs;
        Q.nchunks = (int)st->chunks.size();
        Q.nstages = st->nstages2;
        Q.flush_stages = st->flush_stages;
        Q.stage_bytes = st->stage_bytes2;
        Q.bhalf = st->bhalf;
        Q.table_rows = st->table_rows;
        Q.status = ctx->status_dev;
        TRJ_CUDA_TRY(ctx, cudaFuncSetAttribute(sq_tc2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               st->smem_bytes2));
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3((unsigned)st->grid2);
        cfg.blockDim = dim3(kTcThreads);
        cfg.dynamicSmemBytes = (size_t)st->smem_bytes2;
        cfg.stream = s;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        plan->timer.begin(ctx, s);
        TRJ_CUDA_TRY(ctx, cudaLaunchKernelEx(&cfg, sq_tc2_kernel, st->map_hi, st->map_lo, st->map_hi64, st->map_lo64, Q));
        plan->timer.end(ctx, s);
    } else {
        plan->timer.begin(ctx, s);
        sq_tc_kernel<<<st->grid, k1Threads, st->smem_bytes, s>>>(st->map_hi, st->map_lo, st->map_hi64,
                                                                  st->map_lo64, P);
        plan->timer.end(ctx, s);
    }
    const dim3 rg((unsigned)((st->bmax * 128 + 255) / 256), (unsigned)plan->tiles.size(), (unsigned)plan->nsp);
    tc_reduce_kernel<<<rg, 256, 0, s>>>(st->part, st->acc_stride, st->tiles_dev, plan->tiles_dev, st->chunk_begin_dev,
                                        plan->nsp, plan->tc_out_dev);
    ctx->launches += 3;
    TRJ_CUDA_TRY(ctx, cudaGetLastError());
    return TRJ_OK;
}

extern "C" int trj_sq_plan_set_pairs(trj_sq_plan* plan, int enable) {
    if (!plan) return TRJ_ERR_INVALID;
    TcState* st = reinterpret_cast<TcState*>(plan->tc_state);
    if (st) st->use_pairs = enable ? 1 : 0;
    return TRJ_OK;
}

extern "C" int trj_sq_plan_set_flush(trj_sq_plan* plan, int atoms) {
    if (!plan) return TRJ_ERR_INVALID;
    if (atoms < kStageSlots)
        return trj_fail(plan->ctx, TRJ_ERR_INVALID, "flush interval %d < %d atoms", atoms, kStageSlots);
    TcState* st = reinterpret_cast<TcState*>(plan->tc_state);
    if (st) st->flush_stages = atoms / kStageSlots;
    return TRJ_OK;
}
