// rdf.cu -- species-resolved pair-distance histogram g_ab(r) on sm_100a.
//
// Restates the arithmetic of the reference kernel rdf_sh (src/modules/rdf.cuf:426-487):
// per unordered pair, FP32 minimum image xd -= L*nint(xd/L) per axis, rr2 = (xd^2+yd^2)+zd^2,
// counted when rr2 < side2 into bin nint(sqrt_rn(rr2)/deltar) if 1 <= bin <= lsmax, row
// ind_ij(species_i, species_j).  Every FP32 operation is the explicitly rounded intrinsic
// (__fsub_rn/__fmul_rn/__fadd_rn/__fsqrt_rn/__fdiv_rn), so no FMA contraction changes it.
//
// Unlike the reference's O(N^2) sweep, candidate pairs come from a linked-cell grid:
// cells of edge >= rcut*(1+2^-10), a half-shell stencil (13 neighbour cells + self) so each
// pair is tested once.  The per-pair arithmetic is sign-symmetric (IEEE subtraction, NINT
// half-away-from-zero), so the order (i,j) or (j,i) gives the same rr2 and the same bin;
// the counts equal the all-pairs sweep exactly.  Axes with fewer than 3 cells are not split
// (one cell along that axis); a frame with no split axis is the all-pairs case.
//
// Within a cell, atoms are ordered along a Morton curve over S^3 sub-cells, so the 64 home atoms of
// a warp (two per lane, consecutive in that order) fill a small box.  Each warp tests 32 staged
// neighbour atoms at a time against that box grown by the cutoff (one ballot) and runs the exact
// pair test only for the neighbours that can be in range: a conservative cull, the counts are
// those of the full stencil.
//
// Neighbour-cell atoms are staged into shared memory with 1-D TMA bulk copies
// (cp.async.bulk, no multicast) into two slots, each on its own mbarrier.  Warps walk the task
// sequence independently: the last warp to release a slot refills it with the next task, so there
// is no CTA barrier per task.  Warps count into uint32 shared histogram replicas (warp w uses
// replica w mod nrep); replicas are merged with 64-bit global atomics at exit.
#include <curand_kernel.h>
#include <math.h>

#include <algorithm>
#include <vector>

#include "batch.cuh"
#include "trj_common.cuh"

namespace {

constexpr int kThreads = 256;       // threads per CTA
constexpr int kHomeChunk = 2 * kThreads;  // two home atoms per thread: a warp holds 64 consecutive atoms
constexpr int kJChunk = 512;        // neighbour atoms per staged buffer (8 KB)
constexpr int kSlots = 2;           // staged buffers (tasks in flight per CTA)
constexpr int kMaxOffsets = 14;

struct RdfParams {
    float L[3];
    float h1[3], h2[3];         // |dx| < h1: nint(dx/L) = 0; h1 <= |dx| < h2: +-1; else the division
    float side2, side2_lo, side2_hi;
    float deltar, inv_deltar;
    int lsmax, nsp, nit;
    int floor_bins;             // 0: bin nint(r/deltar) (reference); 1: bin floor(r/deltar)+1
    int nc[3];
    int ncell;
    int noff;
    int hsplit, jsplit;
    int nrep;
    int fast_ok;                // every axis split into >= 5 cells
    float cull2;                // (cutoff * (1 + 2^-10))^2: neighbours farther from a warp's box are skipped
    float cull_pad;             // added to the box half-widths: covers the FP32 rounding of the cull test
    int sbits;                  // sub-cells per cell axis: 2^sbits (Morton order inside a cell)
    long long wait_clocks;      // limit of a warp's wait for a staged neighbour chunk
    int stall_test;             // 1: each warp's first wait is on a barrier nothing arrives on (timeout test)
    int off[kMaxOffsets][3];
    int64_t nitems;
};

struct TaskInfo {
    int sa, na;        // home cell start/count in the sorted array
    int sb;            // first staged neighbour atom (global index into sorted)
    int jcount;        // staged atoms
    int jlocal0;       // index within the neighbour cell of the first staged atom
    int hc;            // home chunk
    int self;          // home cell == neighbour cell
    int fast;          // no minimum image needed for any pair of the task
    int cull;          // both cells hold only coordinates in [-L, L): the box cull applies (wrapped values)
    float img[3];      // periodic image of the neighbour cell: 0 or -+L per axis
    int valid;         // 0 = no more tasks
    int oct;           // 1: warp w's homes are octant w of the home cell (ostart[w] .. ostart[w + 1])
    short ostart[9];   // octant starts within the home cell (oct = 1)
};

__device__ __forceinline__ float min_image_exact(float d, float L) {
    float n = roundf(__fdiv_rn(d, L));
    return __fsub_rn(d, __fmul_rn(L, n));
}

// Minimum image of the reference, d - L*nint(fl(d/L)), without the division below 3L/2: h1 (h2) is the
// least float x >= 0 whose quotient fl(x/L) is >= 1/2 (>= 3/2), found on the host with the same FP32
// division.  Correctly rounded division is monotonic in x, so |d| < h1 <=> nint = 0 and
// h1 <= |d| < h2 <=> nint = +-1 (sign of d): the result is the reference's, bit for bit.
__device__ __forceinline__ float min_image(float d, float L, float h1, float h2) {
    const float a = fabsf(d);
    if (a < h1) return d;
    if (a < h2) return __fsub_rn(d, __fmul_rn(L, copysignf(1.0f, d)));
    return min_image_exact(d, L);  // also NaN
}

// Bin of a pair by the reference's arithmetic (0: not counted).
__device__ __forceinline__ int outcome(float rr2, float side2, float deltar, int lsmax, int floor_bins) {
    if (!(rr2 < side2)) return 0;
    float rr = __fsqrt_rn(rr2);
    float q = __fdiv_rn(rr, deltar);
    int ind = floor_bins ? (int)floorf(q) + 1 : (int)roundf(q);
    return (ind <= lsmax && ind > 0) ? ind : 0;
}

// Task iterator, run by one thread at a time (the thread that refills a slot): items are taken from
// a global counter (dynamic balance); item = (cell, offset, home round, neighbour segment);
// tasks = (home round of up to 512 atoms, neighbour chunk of up to 512 atoms).
struct TaskGen {
    int64_t w;
    int hc, jc;
    int started;
};

__device__ __forceinline__ int wrapc(int c, int n) { return c < 0 ? c + n : (c >= n ? c - n : c); }

// Octant starts of cell c (atoms sa .. sa + na of the sorted array) from the sub-cell starts; returns 1
// when no octant holds more than 64 atoms.  Not inlined: it runs on the refill path only, and its
// loads would otherwise add to the register pressure of the pair loop.
__device__ __noinline__ int octant_starts(const int32_t* __restrict__ fstart, int c, int sa, int na, int sbits,
                                          short* ostart) {
    const int64_t kb = (int64_t)c << (3 * sbits);
    const int step = 1 << (3 * (sbits - 1));
    int mx = 0, prev = 0;
    ostart[0] = 0;
    for (int o = 1; o <= 8; ++o) {
        const int v = o < 8 ? fstart[kb + o * step] - sa : na;
        ostart[o] = (short)v;
        mx = max(mx, v - prev);
        prev = v;
    }
    return mx <= 64;
}

__device__ bool next_task(TaskGen& g, const RdfParams& p, const int32_t* __restrict__ cstart,
                          const int32_t* __restrict__ ccount, const int32_t* __restrict__ cflag,
                          const int32_t* __restrict__ fstart, unsigned long long* work, TaskInfo& t) {
    for (;;) {
        if (!g.started) {
            g.started = 1;
            g.w = (int64_t)atomicAdd(work, 1ull);
            g.hc = -1;
            g.jc = 0;
        }
        if (g.w >= p.nitems) {
            t.valid = 0;
            return false;
        }
        int64_t w = g.w;
        const int seg = (int)(w % p.jsplit);
        w /= p.jsplit;
        const int h = (int)(w % p.hsplit);
        w /= p.hsplit;
        const int o = (int)(w % p.noff);
        const int c = (int)(w / p.noff);
        const int cz = c % p.nc[2];
        const int cy = (c / p.nc[2]) % p.nc[1];
        const int cx = c / (p.nc[2] * p.nc[1]);
        const int ex = cx + p.off[o][0], ey = cy + p.off[o][1], ez = cz + p.off[o][2];
        const int c2 = (wrapc(ex, p.nc[0]) * p.nc[1] + wrapc(ey, p.nc[1])) * p.nc[2] + wrapc(ez, p.nc[2]);
        const int na = ccount[c], nb = ccount[c2];
        const int self = (o == 0);
        if (g.hc < 0) {
            g.hc = h;
            g.jc = 0;
        }
        while (true) {
            if (g.hc * kHomeChunk >= na) break;  // item done
            const int jfirst = self ? g.hc * kHomeChunk : 0;
            const int jtot = nb - jfirst;
            const int s0 = jfirst + (int)((int64_t)jtot * seg / p.jsplit);
            const int s1 = jfirst + (int)((int64_t)jtot * (seg + 1) / p.jsplit);
            const int jstart = s0 + g.jc * kJChunk;
            if (jtot <= 0 || jstart >= s1) {
                g.hc += p.hsplit;
                g.jc = 0;
                continue;
            }
            const bool wraps = ex < 0 || ex >= p.nc[0] || ey < 0 || ey >= p.nc[1] || ez < 0 || ez >= p.nc[2];
            t.sa = cstart[c];
            t.na = na;
            t.sb = cstart[c2] + jstart;
            t.jcount = min(kJChunk, s1 - jstart);
            t.jlocal0 = jstart;
            t.hc = g.hc;
            t.self = self;
            t.fast = p.fast_ok && !wraps && !cflag[c] && !cflag[c2];
            t.cull = !((cflag[c] | cflag[c2]) & 2);
            t.img[0] = ex < 0 ? -p.L[0] : (ex >= p.nc[0] ? p.L[0] : 0.f);
            t.img[1] = ey < 0 ? -p.L[1] : (ey >= p.nc[1] ? p.L[1] : 0.f);
            t.img[2] = ez < 0 ? -p.L[2] : (ez >= p.nc[2] ? p.L[2] : 0.f);
            t.valid = 1;
            // Octant homes: a cell of one home round whose eight Morton octants (sub-cell keys
            // o * 8^(sbits-1) ..) each hold at most 64 atoms gives warp w octant w, a box of half the
            // cell edge, instead of 64 consecutive atoms that may span two octants.
            t.oct = (p.sbits >= 1 && na <= kHomeChunk) ? octant_starts(fstart, c, t.sa, na, p.sbits, t.ostart) : 0;
            g.jc += 1;
            return true;
        }
        g.w = (int64_t)atomicAdd(work, 1ull);
        g.hc = -1;
    }
}

struct PairCounters {
    unsigned long long ulp = 0, fma = 0, counted = 0;
};

// Exact reference outcome of a pair near a bin edge or the cutoff, with its edge statistics:
// returns the bin | 2^29 if a one-ulp change of rr2 changes it | 2^30 if the FMA-contracted rr2
// does.  Scalars by value: nothing of the caller's needs an address (no local-memory copies).
__device__ __noinline__ int exact_bin(float rr2, float x2, float dy, float dz, float side2, float deltar, int lsmax,
                                      int floor_bins) {
    const int ind = outcome(rr2, side2, deltar, lsmax, floor_bins);
    const int olo = outcome(nextafterf(rr2, -INFINITY), side2, deltar, lsmax, floor_bins);
    const int ohi = outcome(nextafterf(rr2, INFINITY), side2, deltar, lsmax, floor_bins);
    const float rr2f = fmaf(dz, dz, fmaf(dy, dy, x2));
    const int fma = outcome(rr2f, side2, deltar, lsmax, floor_bins) != ind;
    return ind | ((olo != ind || ohi != ind) ? (1 << 29) : 0) | (fma ? (1 << 30) : 0);
}

// QMODE: also adds the charge product q_a*q_b of every counted pair to the bin (FP64; the product
// of two FP32 charges is exact in FP64).  rdf.cuf:469-472.
// FLOOR: bins floor(r/deltar)+1 (rdfxy) instead of nint(r/deltar).
template <bool FLOOR, bool QMODE>
__device__ __forceinline__ void bin_pair(float rr2, float x2, float dy, float dz, int row, const RdfParams& p,
                                         unsigned* myhist, PairCounters& pc, double* myq, float qa,
                                         const float* qbp) {
    const float q = rr2 * rsqrtf(rr2) * p.inv_deltar;
    // Nearest integer of q by adding and removing 1.5*2^23 (q < 2^22): qb holds it in its low
    // mantissa bits; d = q - r in [-1/2, 1/2] exactly.
    const float qb = __fadd_rn(q, 12582912.0f);
    const float d = __fsub_rn(q, __fsub_rn(qb, 12582912.0f));
    const float win = fmaf(q, 1.9073486e-6f, 9.5367432e-7f);  // q*2^-19 + 2^-20
    // distance of q from the nearest bin edge: integers (floor bins) or half-integers (nint bins)
    const float edge = FLOOR ? fabsf(d) : 0.5f - fabsf(d);
    int ind;
    if (rr2 >= p.side2_lo || !(edge > win)) {  // NaN (rr2 == 0) takes this path too
        const int e = exact_bin(rr2, x2, dy, dz, p.side2, p.deltar, p.lsmax, p.floor_bins);
        pc.ulp += (e >> 29) & 1;
        pc.fma += (e >> 30) & 1;
        ind = e & ((1 << 29) - 1);
    } else {
        // Away from an edge, round-to-nearest-even and NINT agree, and floor(q) = r - (d < 0).
        const int r = __float_as_int(qb) - 0x4B400000;
        ind = FLOOR ? r + (d > 0.f ? 1 : 0) : r;
        if (ind > p.lsmax) ind = 0;
    }
    if (ind > 0) {
        atomicAdd(&myhist[row * p.lsmax + ind - 1], 1u);
        if (QMODE) atomicAdd(&myq[ind - 1], (double)qa * (double)__ldg(qbp));
    }
}

template <bool FAST, bool FLOOR, bool QMODE>
__device__ __forceinline__ void pair(const float4& a, const float4& b, bool valid, int si, const RdfParams& p,
                                     const int* rowtab, unsigned* myhist, PairCounters& pc, double* myq,
                                     float qa, const float* qbp) {
    float dx = __fsub_rn(b.x, a.x);
    float dy = __fsub_rn(b.y, a.y);
    float dz = __fsub_rn(b.z, a.z);
    if (!FAST) {
        dx = min_image(dx, p.L[0], p.h1[0], p.h2[0]);
        dy = min_image(dy, p.L[1], p.h1[1], p.h2[1]);
        dz = min_image(dz, p.L[2], p.h1[2], p.h2[2]);
    }
    const float x2 = __fmul_rn(dx, dx);
    const float rr2 = __fadd_rn(__fadd_rn(x2, __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    if (valid && rr2 < p.side2_hi) {
        const int sj = __float_as_int(b.w);
        if ((unsigned)sj < (unsigned)p.nsp)
            bin_pair<FLOOR, QMODE>(rr2, x2, dy, dz, rowtab[si * p.nsp + sj], p, myhist, pc, myq, qa, qbp);
    }
}

// Box of the warp's home atoms, centred on the neighbour cell's periodic image: a neighbour b can be
// within the cutoff of some home atom only if |b - c| - h, clipped at 0 per axis, has squared length
// <= cull2.  Unsplit axes (one cell) get an infinite half-width: no cull along them.
struct WarpBox {
    float4 c, h;  // centre (x, y, z) and half-widths (x, y, z); .w unused
};

__device__ __forceinline__ void axis_box(float v0, bool has0, float v1, bool has1, bool split, float img, float pad,
                                         float& c, float& h) {
    // Wrapped coordinates of cull tasks lie in [0, L]: their bit patterns order like the values (+0 for -0).
    const unsigned b0 = __float_as_uint(v0 + 0.0f), b1 = __float_as_uint(v1 + 0.0f);
    const unsigned lo = min(has0 ? b0 : 0x7f800000u, has1 ? b1 : 0x7f800000u);
    const unsigned hi = max(has0 ? b0 : 0u, has1 ? b1 : 0u);
    const float mn = __uint_as_float(__reduce_min_sync(0xffffffffu, lo));
    const float mx = __uint_as_float(__reduce_max_sync(0xffffffffu, hi));
    c = 0.5f * (mn + mx) - img;
    h = split ? 0.5f * (mx - mn) + pad : INFINITY;
}

// Wrapped coordinate of a folded one in [-L, L): x, or x + L for x < 0 (the same FP32 value the cell
// assignment computes, so the atom lies in its cell's range).  The fold of select_ncdfinput keeps
// negative coordinates negative; the cull works on the wrapped values.
__device__ __forceinline__ float wrap_cull(float x, float L) { return x < 0.f ? __fadd_rn(x, L) : x; }

__device__ __forceinline__ bool maybe_near(const float4& b, const float4& c, const float4& h, float cull2,
                                           const float (&L)[3]) {
    const float gx = fmaxf(fabsf(wrap_cull(b.x, L[0]) - c.x) - h.x, 0.f);
    const float gy = fmaxf(fabsf(wrap_cull(b.y, L[1]) - c.y) - h.y, 0.f);
    const float gz = fmaxf(fabsf(wrap_cull(b.z, L[2]) - c.z) - h.z, 0.f);
    return fmaf(gz, gz, fmaf(gy, gy, gx * gx)) <= cull2;
}

// One task for one warp: its 64 home atoms (a0 = atom il0, a1 = atom il0 + 32 per lane) against the
// staged neighbour chunk.  Blocks of 32 neighbours are culled against the warp's box (kept in shared
// memory, `wb`) with one ballot; the survivors are tested exactly.  Returns the candidate pairs tested.
// Lanes whose bit index k has jj0 + k > lim: the neighbours of a block that pair with a home.
__device__ __forceinline__ unsigned after_mask(int lim, int jj0) {
    const int s = lim - jj0;
    return s < 0 ? 0xffffffffu : (s >= 31 ? 0u : (0xffffffffu << (s + 1)));
}

// SELF: home and neighbour cell are the same cell (pairs need j > i within it).
template <bool FAST, bool SELF, bool FLOOR, bool QMODE>
__device__ __forceinline__ unsigned run_task(const TaskInfo& ti, const float4* __restrict__ bj, const float4& a0,
                                             const float4& a1, bool h0, bool h1, int il0, int il0w, int s0, int s1,
                                             unsigned lane, const RdfParams& p, const int* rowtab, unsigned* myhist,
                                             PairCounters& pc, double* myq, float qa0, float qa1, const float* qj,
                                             WarpBox* wb) {
    if (ti.cull) {
        float cx, cy, cz, hx, hy, hz;
        axis_box(wrap_cull(a0.x, p.L[0]), h0, wrap_cull(a1.x, p.L[0]), h1, p.nc[0] > 1, ti.img[0], p.cull_pad, cx, hx);
        axis_box(wrap_cull(a0.y, p.L[1]), h0, wrap_cull(a1.y, p.L[1]), h1, p.nc[1] > 1, ti.img[1], p.cull_pad, cy, hy);
        axis_box(wrap_cull(a0.z, p.L[2]), h0, wrap_cull(a1.z, p.L[2]), h1, p.nc[2] > 1, ti.img[2], p.cull_pad, cz, hz);
        if (lane == 0) {
            wb->c = make_float4(cx, cy, cz, 0.f);
            wb->h = make_float4(hx, hy, hz, 0.f);
        }
        __syncwarp();
    }
    const int jbeg = SELF ? max(0, il0w + 1 - ti.jlocal0) : 0;
    const int lim0 = SELF ? il0 - ti.jlocal0 : -1;  // a0 pairs need jj > lim0
    const int lim1 = SELF ? lim0 + 32 : -1;         // a1 pairs need jj > lim1
    unsigned tested = 0;
    for (int jj0 = jbeg; jj0 < ti.jcount; jj0 += 32) {
        const int jl = jj0 + (int)lane;
        bool keep = jl < ti.jcount;
        if (ti.cull && keep) keep = maybe_near(bj[jl], wb->c, wb->h, p.cull2, p.L);
        unsigned m = __ballot_sync(0xffffffffu, keep);
        if (SELF)
            tested += (h0 ? __popc(m & after_mask(lim0, jj0)) : 0) + (h1 ? __popc(m & after_mask(lim1, jj0)) : 0);
        else
            tested += __popc(m) * ((unsigned)h0 + (unsigned)h1);
        while (m) {
            const int k0 = __ffs(m) - 1;
            m &= m - 1u;
            const int j0 = jj0 + k0;
            const float4 b0 = bj[j0];
            pair<FAST, FLOOR, QMODE>(a0, b0, SELF ? (h0 && j0 > lim0) : h0, s0, p, rowtab, myhist, pc, myq, qa0,
                                     qj + j0);
            pair<FAST, FLOOR, QMODE>(a1, b0, SELF ? (h1 && j0 > lim1) : h1, s1, p, rowtab, myhist, pc, myq, qa1,
                                     qj + j0);
        }
    }
    return tested;
}

// Arms the next phase of a staging slot: the next task's neighbour chunk by bulk copy, or a plain
// arrival with valid = 0 when the work is exhausted (readers of that phase leave the task loop).
__device__ __forceinline__ void refill_slot(int slot, TaskGen& gen, const RdfParams& p,
                                            const int32_t* __restrict__ cstart, const int32_t* __restrict__ ccount,
                                            const int32_t* __restrict__ cflag, const int32_t* __restrict__ fstart,
                                            unsigned long long* work,
                                            const float4* __restrict__ sorted, TaskInfo* tinfo, uint64_t* bars,
                                            unsigned* phases, float4* buf) {
    TaskInfo nx;
    const bool ok = next_task(gen, p, cstart, ccount, cflag, fstart, work, nx);
    tinfo[slot] = nx;
    phases[slot] += 1u;
    if (ok) {
        // The slot's previous contents were read through the generic proxy; order those reads before
        // the bulk copy (async proxy) overwrites them.
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        trj_mbar_arrive_expect_tx(&bars[slot], nx.jcount * 16u);
        trj_bulk_g2s(buf + slot * kJChunk, sorted + nx.sb, nx.jcount * 16u, &bars[slot]);
    } else {
        trj_mbar_arrive(&bars[slot]);
    }
}

// QMODE: sorted_q holds the charges in cell order and gqq_frame (lsmax doubles) receives this
// frame's sum of q_a*q_b per bin; the charge replicas (lsmax doubles each, warp w uses w mod nrep)
// follow the count replicas in shared memory.
template <bool FLOOR, bool QMODE>
__global__ void __launch_bounds__(kThreads, 4) rdf_pairs_kernel(RdfParams p, const float4* __restrict__ sorted,
                                                             const int32_t* __restrict__ cstart,
                                                             const int32_t* __restrict__ ccount,
                                                             const int32_t* __restrict__ cflag,
                                                             const int32_t* __restrict__ fstart,
                                                             unsigned long long* __restrict__ work,
                                                             unsigned long long* __restrict__ hist_g,
                                                             unsigned long long* __restrict__ edge_g,
                                                             unsigned* __restrict__ status,
                                                             const float* __restrict__ sorted_q,
                                                             double* __restrict__ gqq_frame) {
    extern __shared__ __align__(128) unsigned char smem[];
    float4* buf = reinterpret_cast<float4*>(smem);                       // [kSlots][kJChunk]
    unsigned* hist = reinterpret_cast<unsigned*>(smem + kSlots * kJChunk * sizeof(float4));
    __shared__ __align__(8) uint64_t bars[kSlots];
    __shared__ __align__(8) uint64_t never;  // no thread arrives on it: the target of the stall test
    __shared__ TaskInfo tinfo[kSlots];
    __shared__ unsigned released[kSlots];  // warps done with the slot's task
    __shared__ unsigned phases[kSlots];    // phases armed per slot
    __shared__ TaskGen gen;                // task iterator, used by one refilling thread at a time
    __shared__ int rowtab[16 * 16];
    __shared__ int abort_flag;
    __shared__ WarpBox wboxes[kThreads / 32];

    const int tid = threadIdx.x, warp = tid / 32;
    const unsigned lane = (unsigned)tid & 31u;
    const int hsz = p.nit * p.lsmax;
    unsigned* myhist = hist + (size_t)(warp % p.nrep) * hsz;
    for (int k = tid; k < p.nrep * hsz; k += blockDim.x) hist[k] = 0u;
    double* qhist = nullptr;
    double* myq = nullptr;
    if (QMODE) {
        qhist = reinterpret_cast<double*>(hist + (((size_t)p.nrep * hsz + 1) & ~(size_t)1));
        myq = qhist + (size_t)(warp % p.nrep) * p.lsmax;
        for (int k = tid; k < p.nrep * p.lsmax; k += blockDim.x) qhist[k] = 0.0;
    }
    for (int k = tid; k < p.nsp * p.nsp; k += blockDim.x) rowtab[k] = trj_pair_row(k / p.nsp, k % p.nsp, p.nsp);
    if (tid == 0) {
        gen.started = 0;
        abort_flag = 0;
        for (int sl = 0; sl < kSlots; ++sl) {
            trj_mbar_init(&bars[sl], 1);
            released[sl] = 0u;
            phases[sl] = 0u;
        }
        trj_mbar_init(&never, 1);
        trj_fence_mbar_init();
        for (int sl = 0; sl < kSlots; ++sl) refill_slot(sl, gen, p, cstart, ccount, cflag, fstart, work, sorted, tinfo, bars, phases, buf);
    }
    __syncthreads();
    PairCounters pc;
    unsigned long long n_tested = 0;
    // Warps walk the task sequence independently: task t sits in slot t % kSlots; the last warp to
    // release a slot refills it with the next task, so a warp may run up to kSlots - 1 tasks ahead of
    // the slowest one instead of meeting it at a CTA barrier after every task.
    for (int t = 0;; ++t) {
        const int slot = t % kSlots;
        if (__shfl_sync(0xffffffffu, *(volatile int*)&abort_flag, 0)) break;  // warp-uniform
        // Warp-uniform outcome: the task loop below uses full-warp ballots.
        const bool stall = p.stall_test && t == 0;
        if (!__all_sync(0xffffffffu, trj_mbar_wait_limit(stall ? &never : &bars[slot],
                                                         stall ? 0u : (unsigned)(t / kSlots) & 1u,
                                                         p.wait_clocks))) {
            if (lane == 0) {
                trj_raise(status, TRJ_DEV_TIMEOUT);
                *(volatile int*)&abort_flag = 1;
            }
            break;
        }
        const TaskInfo ti = tinfo[slot];
        if (!ti.valid) break;
        // The warp's home atoms [hbeg, hend) within the cell: its octant, or 64 consecutive atoms of the round.
        const int hbeg = ti.oct ? (int)tinfo[slot].ostart[warp] : ti.hc * kHomeChunk + 64 * warp;
        const int hend = ti.oct ? (int)tinfo[slot].ostart[warp + 1] : min(ti.na, hbeg + 64);
        const int il0 = hbeg + (int)lane, il1 = il0 + 32;
        const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 a0 = il0 < hend ? sorted[ti.sa + il0] : z4;
        const float4 a1 = il1 < hend ? sorted[ti.sa + il1] : z4;
        const int s0 = __float_as_int(a0.w), s1 = __float_as_int(a1.w);
        // A species outside 0..nsp-1 can only come from a frame already flagged as bad data.
        const bool h0 = il0 < hend && (unsigned)s0 < (unsigned)p.nsp;
        const bool h1 = il1 < hend && (unsigned)s1 < (unsigned)p.nsp;
        const float qa0 = (QMODE && il0 < hend) ? sorted_q[ti.sa + il0] : 0.f;
        const float qa1 = (QMODE && il1 < hend) ? sorted_q[ti.sa + il1] : 0.f;
        const float* qj = QMODE ? sorted_q + ti.sb : nullptr;
        const float4* bj = buf + slot * kJChunk;
        WarpBox* wb = &wboxes[warp];
#define TRJ_RUN(F, S)                                                                                       \
    run_task<F, S, FLOOR, QMODE>(ti, bj, a0, a1, h0, h1, il0, hbeg, s0, s1, lane, p, rowtab, myhist, pc, myq, qa0, \
                                 qa1, qj, wb)
        if (hbeg < hend) {  // warp-uniform: the warp has home atoms in this task
            if (ti.fast)
                n_tested += ti.self ? TRJ_RUN(true, true) : TRJ_RUN(true, false);
            else
                n_tested += ti.self ? TRJ_RUN(false, true) : TRJ_RUN(false, false);
        }
#undef TRJ_RUN
        // Release the slot; the last warp refills it.
        __syncwarp();
        if (lane == 0) {
            __threadfence_block();
            if (atomicAdd(&released[slot], 1u) == kThreads / 32 - 1) {
                released[slot] = 0u;
                __threadfence_block();
                refill_slot(slot, gen, p, cstart, ccount, cflag, fstart, work, sorted, tinfo, bars, phases, buf);
            }
        }
        __syncwarp();
    }
    __syncthreads();
    if (tid == 0 && abort_flag) {
        // Let copies still in flight land before the CTA exits (bounded by the default limit, not by
        // the plan's wait limit: a copy always lands).
        for (int sl = 0; sl < kSlots; ++sl)
            if (phases[sl]) trj_mbar_wait(&bars[sl], (phases[sl] - 1) & 1);
    }
    __syncthreads();
    // Merge replicas into the global uint64 histogram (their total is the counted pairs).
    for (int k = tid; k < hsz; k += blockDim.x) {
        unsigned long long s = 0;
        for (int r = 0; r < p.nrep; ++r) s += hist[(size_t)r * hsz + k];
        if (s) atomicAdd(&hist_g[k], s);
        pc.counted += s;
    }
    if (QMODE) {
        for (int k = tid; k < p.lsmax; k += blockDim.x) {
            double s = 0.0;
            for (int r = 0; r < p.nrep; ++r) s += qhist[(size_t)r * p.lsmax + k];
            if (s != 0.0) atomicAdd(&gqq_frame[k], s);
        }
    }
    if (edge_g) {
        unsigned long long n_ulp = pc.ulp, n_fma = pc.fma, n_counted = pc.counted;
        for (int off = 16; off > 0; off >>= 1) {
            n_ulp += __shfl_down_sync(0xffffffffu, n_ulp, off);
            n_fma += __shfl_down_sync(0xffffffffu, n_fma, off);
            n_counted += __shfl_down_sync(0xffffffffu, n_counted, off);
            n_tested += __shfl_down_sync(0xffffffffu, n_tested, off);
        }
        if ((tid & 31) == 0) {
            if (n_ulp) atomicAdd(&edge_g[TRJ_EDGE_ULP], n_ulp);
            if (n_fma) atomicAdd(&edge_g[TRJ_EDGE_FMA], n_fma);
            if (n_counted) atomicAdd(&edge_g[TRJ_EDGE_COUNTED], n_counted);
            if (n_tested) atomicAdd(&edge_g[TRJ_EDGE_TESTED], n_tested);
        }
    }
}

// Cell of each atom from its wrapped coordinate, and its sub-cell: the cell is split into
// 2^sbits parts per axis and the parts are numbered along a Morton curve (bits interleaved x, y, z
// from the lowest), so atoms sorted by key = cell * 8^sbits + sub-cell are cell-contiguous and
// spatially ordered inside each cell.  Per-key and per-cell counts, per-key slots.
__global__ void cell_assign_kernel(const float4* __restrict__ packed, int64_t n, float Lx, float Ly,
                                   float Lz, int ncx, int ncy, int ncz, int sbits, int32_t* __restrict__ fcount,
                                   int32_t* __restrict__ ccount, int32_t* __restrict__ cflag,
                                   int32_t* __restrict__ akey, int32_t* __restrict__ aslot) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = packed[i];
    float L[3] = {Lx, Ly, Lz};
    int nc[3] = {ncx, ncy, ncz};
    float r[3] = {v.x, v.y, v.z};
    int k[3], sub[3];
    const int S = 1 << sbits;
    bool outside = false, far = false;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        outside |= !(r[d] >= 0.0f && r[d] < L[d]);
        far |= !(r[d] >= -L[d] && r[d] < L[d]);
        float w = r[d] - L[d] * floorf(r[d] / L[d]);
        float t = w * ((float)nc[d] / L[d]);
        int c = (int)t;
        c = c < 0 ? 0 : (c >= nc[d] ? nc[d] - 1 : c);
        k[d] = c;
        int sc = (int)((t - (float)c) * (float)S);
        sub[d] = sc < 0 ? 0 : (sc >= S ? S - 1 : sc);  // also catches NaN coordinates (sc = 0)
    }
    int m = 0;
    for (int b = 0; b < sbits; ++b)
        m |= (((sub[0] >> b) & 1) << (3 * b)) | (((sub[1] >> b) & 1) << (3 * b + 1)) |
             (((sub[2] >> b) & 1) << (3 * b + 2));
    int c = (k[0] * ncy + k[1]) * ncz + k[2];
    const int key = (c << (3 * sbits)) | m;
    akey[i] = key;
    aslot[i] = atomicAdd(&fcount[key], 1);
    atomicAdd(&ccount[c], 1);
    // bit 0: a coordinate outside [0, L) (pairs of the cell need the minimum image);
    // bit 1: a coordinate outside [-L, L) or NaN (its wrapped value is not x or x + L: no box cull)
    if (outside) atomicOr(&cflag[c], far ? 3 : 1);
}

// Start of every (cell, sub-cell) key: the cell's start plus the exclusive prefix of its sub-cell
// counts.  One warp per cell.
__global__ void sub_offsets_kernel(const int32_t* __restrict__ fcount, const int32_t* __restrict__ cstart, int ncell,
                                   int sbits, int32_t* __restrict__ fstart) {
    const int c = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const unsigned lane = threadIdx.x & 31u;
    if (c >= ncell) return;
    const int nsub = 1 << (3 * sbits);
    const int64_t base = (int64_t)c << (3 * sbits);
    int carry = cstart[c];
    for (int s0 = 0; s0 < nsub; s0 += 32) {
        const int s = s0 + (int)lane;
        const int v = s < nsub ? fcount[base + s] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if ((int)lane >= o) x += y;
        }
        if (s < nsub) fstart[base + s] = carry + x - v;
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
}

__global__ void cell_scatter_kernel(const float4* __restrict__ packed, int64_t n,
                                    const int32_t* __restrict__ akey, const int32_t* __restrict__ aslot,
                                    const int32_t* __restrict__ fstart, float4* __restrict__ sorted,
                                    const float* __restrict__ q, float* __restrict__ sorted_q) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t d = fstart[akey[i]] + aslot[i];
    sorted[d] = packed[i];
    if (q) sorted_q[d] = q[i];
}

// One block, after the pair kernel: avq2 = sum(q^2)/N in FP64 rounded to FP32 (rdf.cuf:272, where
// avq2 is a default-real variable), then gqq += gqq_frame/avq2 (rdf.cuf:273).  The reduction order
// is fixed, so avq2 does not depend on scheduling.
__global__ void gqq_finish_kernel(const float* __restrict__ q, int64_t n, const double* __restrict__ gqq_frame,
                                  int lsmax, double* __restrict__ gqq) {
    __shared__ double part[1024];
    double s = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = (double)q[i];
        s += v * v;
    }
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off) part[threadIdx.x] += part[threadIdx.x + off];
        __syncthreads();
    }
    const float avq2 = (float)(part[0] / (double)n);
    for (int k = threadIdx.x; k < lsmax; k += blockDim.x) gqq[k] += gqq_frame[k] / (double)avq2;
}

// Single-block exclusive scan of int32 counts (length up to a few million).
__global__ void scan_exclusive_kernel(const int32_t* __restrict__ in, int32_t* __restrict__ out, int n) {
    __shared__ int32_t part[1024];
    int per = (n + blockDim.x - 1) / blockDim.x;
    int b0 = threadIdx.x * per, b1 = min(n, b0 + per);
    int32_t s = 0;
    for (int k = b0; k < b1; ++k) s += in[k];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < (int)blockDim.x; off <<= 1) {
        int32_t v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int32_t run = part[threadIdx.x] - s;
    for (int k = b0; k < b1; ++k) {
        out[k] = run;
        run += in[k];
    }
    if (threadIdx.x == blockDim.x - 1) out[n] = part[threadIdx.x];
}

// Number fluctuations (s2D3_sh, rdf.cuf:489-553): block b draws one point uniformly in the box with
// the reference's generator and seed (XORWOW, curand_init(b + 12345, 0, 0), b 1-based), counts the
// atoms within each radius r_k = k*deltar (cumulative over nint(r/deltar) bins, the reference's
// gi_s(ind:lsmax) += 1) from the cells around it, and adds N_k and N_k^2 to the int64 sums.
__global__ void s2n_kernel(const float4* __restrict__ sorted, const int32_t* __restrict__ cstart,
                           const int32_t* __restrict__ ccount, float Lx, float Ly, float Lz, int ncx, int ncy,
                           int ncz, float side2, float deltar, int lsmax, unsigned long long* __restrict__ gi,
                           unsigned long long* __restrict__ g2i, float* __restrict__ points, int dim) {
    extern __shared__ unsigned long long cnt[];  // lsmax + 1
    __shared__ float pt[3];
    for (int k = threadIdx.x; k <= lsmax; k += blockDim.x) cnt[k] = 0ull;
    if (threadIdx.x == 0) {
        curandStateXORWOW_t h;
        curand_init((unsigned long long)blockIdx.x + 1ull + 12345ull, 0ull, 0ull, &h);
        pt[0] = Lx * curand_uniform(&h);
        pt[1] = Ly * curand_uniform(&h);
        pt[2] = dim == 2 ? 0.f : Lz * curand_uniform(&h);  // s2D2_sh draws x and y only (rdf.cuf:580-581)
        if (points) {
            points[3 * blockIdx.x] = pt[0];
            points[3 * blockIdx.x + 1] = pt[1];
            points[3 * blockIdx.x + 2] = pt[2];
        }
    }
    __syncthreads();
    const float L[3] = {Lx, Ly, Lz};
    const int nc[3] = {ncx, ncy, ncz};
    int pc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {  // the point's cell, as cell_assign_kernel bins an atom
        const float w = pt[d] - L[d] * floorf(pt[d] / L[d]);
        int c = (int)(w * ((float)nc[d] / L[d]));
        pc[d] = c < 0 ? 0 : (c >= nc[d] ? nc[d] - 1 : c);
    }
    const int rx = ncx > 1 ? 1 : 0, ry = ncy > 1 ? 1 : 0, rz = ncz > 1 ? 1 : 0;
    for (int dx = -rx; dx <= rx; ++dx)
        for (int dy = -ry; dy <= ry; ++dy)
            for (int dz = -rz; dz <= rz; ++dz) {
                const int cx = (pc[0] + dx + ncx) % ncx, cy = (pc[1] + dy + ncy) % ncy, cz = (pc[2] + dz + ncz) % ncz;
                const int c = (cx * ncy + cy) * ncz + cz;
                const int a0 = cstart[c], na = ccount[c];
                for (int j = threadIdx.x; j < na; j += blockDim.x) {
                    const float4 a = sorted[a0 + j];
                    // rdf.cuf:533-541: difference point - atom, minimum image, (x^2 + y^2) + z^2, FP32
                    float xd = __fsub_rn(pt[0], a.x), yd = __fsub_rn(pt[1], a.y), zd = __fsub_rn(pt[2], a.z);
                    xd = __fsub_rn(xd, __fmul_rn(Lx, roundf(__fdiv_rn(xd, Lx))));
                    yd = __fsub_rn(yd, __fmul_rn(Ly, roundf(__fdiv_rn(yd, Ly))));
                    zd = __fsub_rn(zd, __fmul_rn(Lz, roundf(__fdiv_rn(zd, Lz))));
                    const float rr2 = __fadd_rn(__fadd_rn(__fmul_rn(xd, xd), __fmul_rn(yd, yd)), __fmul_rn(zd, zd));
                    if (rr2 < side2) {
                        const int ind = (int)roundf(__fdiv_rn(__fsqrt_rn(rr2), deltar));
                        if (ind >= 0 && ind <= lsmax) atomicAdd(&cnt[ind], 1ull);
                    }
                }
            }
    __syncthreads();
    if (threadIdx.x == 0) {  // cumulative counts N_k = sum_{j <= k} cnt[j]
        unsigned long long run = 0;
        for (int k = 0; k <= lsmax; ++k) {
            run += cnt[k];
            cnt[k] = run;
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k <= lsmax; k += blockDim.x) {
        const unsigned long long v = cnt[k];
        if (v) {
            atomicAdd(&gi[k], v);
            atomicAdd(&g2i[k], v * v);
        }
    }
}


// ---- fused multi-request launch: all-pairs histogram of every packed frame ---------------------
//
// Unit = (item, tile pair bi <= bj) of kBatchTile x kBatchTile atoms of one frame: home atom
// i = bi * 256 + thread against the staged tile bj (j > i on the diagonal tile), each pair through the
// general path of the cell kernel (reference minimum image, exact binning near edges), so the counts
// are those of the reference's all-pairs sweep (rdf.cuf:449-475).  Units come from a global counter;
// a CTA keeps the counts of one item in two shared replicas (even and odd warps) and merges them into
// that item's uint64 histogram when its next unit belongs to another item, and at exit.
template <bool FLOOR>
__device__ __forceinline__ unsigned batch_tile_pairs(const float4* __restrict__ tile, int jcount, const float4& a,
                                                     bool has_a, int il, bool diag, int si, const RdfParams& P,
                                                     const int* rowtab, unsigned* myhist, PairCounters& pc) {
    unsigned tested = 0;
    for (int jj = 0; jj < jcount; ++jj) {
        const bool valid = has_a && (!diag || jj > il);
        tested += valid ? 1u : 0u;
        pair<false, FLOOR, false>(a, tile[jj], valid, si, P, rowtab, myhist, pc, nullptr, 0.f, nullptr);
    }
    return tested;
}

__device__ __forceinline__ void batch_pairs_flush(const BatchItem& it, unsigned* hist, int hist_words,
                                                  PairCounters& pc, unsigned long long& tested) {
    const int hsz = it.nit * it.lsmax;
    for (int k = threadIdx.x; k < hsz; k += kBatchThreads) {
        const unsigned long long v = (unsigned long long)hist[k] + hist[hist_words + k];
        if (v) atomicAdd(&it.hist[k], v);
        pc.counted += v;
        hist[k] = 0u;
        hist[hist_words + k] = 0u;
    }
    if (it.edge) {
        unsigned long long n_ulp = pc.ulp, n_fma = pc.fma, n_counted = pc.counted, n_tested = tested;
        for (int off = 16; off > 0; off >>= 1) {
            n_ulp += __shfl_down_sync(0xffffffffu, n_ulp, off);
            n_fma += __shfl_down_sync(0xffffffffu, n_fma, off);
            n_counted += __shfl_down_sync(0xffffffffu, n_counted, off);
            n_tested += __shfl_down_sync(0xffffffffu, n_tested, off);
        }
        if ((threadIdx.x & 31) == 0) {
            if (n_ulp) atomicAdd(&it.edge[TRJ_EDGE_ULP], n_ulp);
            if (n_fma) atomicAdd(&it.edge[TRJ_EDGE_FMA], n_fma);
            if (n_counted) atomicAdd(&it.edge[TRJ_EDGE_COUNTED], n_counted);
            if (n_tested) atomicAdd(&it.edge[TRJ_EDGE_TESTED], n_tested);
        }
    }
    pc = PairCounters();
    tested = 0;
}

__global__ void __launch_bounds__(kBatchThreads, 3) batch_pairs_kernel(BatchHeader* __restrict__ hdr,
                                                                    const BatchItem* __restrict__ items,
                                                                    const float4* __restrict__ packed,
                                                                    int hist_words) {
    extern __shared__ __align__(128) unsigned char smem[];
    float4* tile = reinterpret_cast<float4*>(smem);                              // [kBatchTile]
    unsigned* hist = reinterpret_cast<unsigned*>(smem + kBatchTile * sizeof(float4));  // [2][hist_words]
    __shared__ int rowtab[kBatchMaxSpecies * kBatchMaxSpecies];
    __shared__ long long unit_s;
    const int tid = threadIdx.x;
    unsigned* myhist = hist + ((tid >> 5) & 1) * hist_words;
    for (int k = tid; k < 2 * hist_words; k += kBatchThreads) hist[k] = 0u;
    const int nitems = hdr->nitems;
    const int64_t total = hdr->total_pair;
    int cur = -1;
    RdfParams P;
    int n = 0, ntile = 0;
    int64_t off = 0;
    PairCounters pc;
    unsigned long long tested = 0;
    while (true) {
        if (tid == 0) unit_s = (long long)atomicAdd(&hdr->counter[0], 1ull);
        __syncthreads();
        const int64_t u = unit_s;
        const int r = u < total ? batch_item_of<&BatchItem::pair_begin>(items, nitems, u) : -1;
        if (r != cur) {  // block-uniform
            if (cur >= 0) batch_pairs_flush(items[cur], hist, hist_words, pc, tested);
            cur = r;
            if (r >= 0) {
                const BatchItem& it = items[r];
                for (int d = 0; d < 3; ++d) {
                    P.L[d] = it.L[d];
                    P.h1[d] = it.h1[d];
                    P.h2[d] = it.h2[d];
                }
                P.side2 = it.side2;
                P.side2_lo = it.side2_lo;
                P.side2_hi = it.side2_hi;
                P.deltar = it.deltar;
                P.inv_deltar = it.inv_deltar;
                P.lsmax = it.lsmax;
                P.nsp = it.nsp;
                P.nit = it.nit;
                P.floor_bins = it.floor_bins;
                n = it.n;
                ntile = it.ntile;
                off = it.atom_off;
                for (int k = tid; k < P.nsp * P.nsp; k += kBatchThreads)
                    rowtab[k] = trj_pair_row(k / P.nsp, k % P.nsp, P.nsp);
            }
            __syncthreads();
        }
        if (r < 0) break;
        // tile pair (bi, bj), bi <= bj, of triangle index t (row bi holds ntile - bi pairs)
        const int64_t t = u - items[r].pair_begin;
        const double b2 = 2.0 * ntile + 1.0;
        int bi = (int)((b2 - sqrt(b2 * b2 - 8.0 * (double)t)) * 0.5);
        auto row_start = [&](int b) { return (int64_t)b * ntile - (int64_t)b * (b - 1) / 2; };
        while (bi > 0 && row_start(bi) > t) --bi;
        while (bi + 1 < ntile && row_start(bi + 1) <= t) ++bi;
        const int bj = bi + (int)(t - row_start(bi));
        const int j = bj * kBatchTile + tid;
        tile[tid] = j < n ? packed[off + j] : make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
        const int i = bi * kBatchTile + tid;
        const float4 a = i < n ? packed[off + i] : make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
        const int si = __float_as_int(a.w);
        const bool has_a = i < n && (unsigned)si < (unsigned)P.nsp;
        const int jcount = min(kBatchTile, n - bj * kBatchTile);
        __syncthreads();
        tested += P.floor_bins
                      ? batch_tile_pairs<true>(tile, jcount, a, has_a, tid, bi == bj, si, P, rowtab, myhist, pc)
                      : batch_tile_pairs<false>(tile, jcount, a, has_a, tid, bi == bj, si, P, rowtab, myhist, pc);
        __syncthreads();
    }
}

}  // namespace

struct trj_rdf_plan {
    trj_ctx* ctx = nullptr;
    int nsp = 0, nit = 0, lsmax = 0;
    int floor_bins = 0;
    long long wait_clocks = TRJ_WAIT_CLOCKS;  // limit of the pair kernel's waits for staged chunks
    int stall_test = 0;
    int dim = 3;                // 2: frames in the xy plane (z = 0); z is neither clipped nor split
    float deltar = 0.f, rcrdf_eff = 0.f, side2 = 0.f;
    int64_t n_max = 0;
    int ncell_cap = 0;
    int nc[3] = {1, 1, 1};
    int32_t* ccount = nullptr;  // ncell_cap
    int32_t* cflag = nullptr;   // ncell_cap: bit 0 a coordinate outside [0, L), bit 1 outside [-L, L)
    unsigned long long* work = nullptr;  // item counter of the pair kernel
    int32_t* cstart = nullptr;  // ncell_cap + 1
    int64_t fine_cap = 0;       // capacity of the per-(cell, sub-cell) arrays
    int32_t* fcount = nullptr;  // fine_cap
    int32_t* fstart = nullptr;  // fine_cap + 1
    int32_t* akey = nullptr;    // n_max: (cell, sub-cell) key per atom
    int32_t* aslot = nullptr;   // n_max
    float4* sorted = nullptr;   // n_max
    float* sorted_q = nullptr;  // n_max charges in cell order (first charged call)
    int cells_valid = 0;        // sorted/cstart/ccount hold the last accumulated frame
    float box_last[3] = {0.f, 0.f, 0.f};
    double* gqq_frame = nullptr;  // lsmax: this frame's charge-product sums
    int64_t scratch_bytes = 0;
    trj_kernel_timer timer;
};

// Least float x >= 0 with fl(x / L) >= q in FP32 (host SSE division, correctly rounded like the
// device's __fdiv_rn): the minimum-image thresholds of min_image.
static float nint_threshold(float L, float q) {
    volatile float vl = L;  // keep the division in single precision at run time
    float x = q * L;
    for (int k = 0; k < 256 && x > 0.f && x / vl >= q; ++k) x = nextafterf(x, 0.f);
    for (int k = 0; k < 256 && x / vl < q; ++k) x = nextafterf(x, INFINITY);
    return x;
}

static int nint_host(float x) {  // Fortran NINT: half away from zero
    double v = (double)x;
    return (int)(v >= 0 ? floor(v + 0.5) : -floor(-v + 0.5));
}

// Smallest box edge of the plan's geometry (the x and y edges in 2D).
static float min_edge(const float box[3], int dim) {
    return dim == 2 ? fminf(box[0], box[1]) : fminf(box[0], fminf(box[1], box[2]));
}

// Cells per axis for cutoff^2 side2 in box L; axes with < 3 cells are not split (nor z in 2D).
static void cells_for(const float L[3], float side2, int nc[3], int dim = 3) {
    double rc = sqrt((double)side2) * (1.0 + 1.0 / 1024.0);
    for (int d = 0; d < 3; ++d) {
        int k = rc > 0 ? (int)floor((double)L[d] / rc) : 1;
        if (k < 3) k = 1;
        if (k > 1024) k = 1024;
        nc[d] = k;
    }
    if (dim == 2) nc[2] = 1;
}

static int rdf_plan_create_impl(trj_ctx* ctx, int nsp, float deltar, float rcrdf, const float box[3],
                                int64_t n_max, int dim, trj_rdf_plan** out) {
    if (!ctx || !out || !box) return TRJ_ERR_INVALID;
    *out = nullptr;
    if (nsp < 1 || nsp > 16) return trj_fail(ctx, TRJ_ERR_INVALID, "rdf plan: nsp=%d (1..16)", nsp);
    if (!(deltar > 0.f)) return trj_fail(ctx, TRJ_ERR_INVALID, "rdf plan: deltar must be > 0");
    if (!(box[0] > 0.f && box[1] > 0.f && box[2] > 0.f))
        return trj_fail(ctx, TRJ_ERR_INVALID, "rdf plan: box edges must be positive");
    if (n_max < 0 || n_max > (int64_t)INT32_MAX)
        return trj_fail(ctx, TRJ_ERR_INVALID, "rdf plan: n_max out of range");
    trj_rdf_plan* p = new trj_rdf_plan();
    p->ctx = ctx;
    p->nsp = nsp;
    p->nit = nsp * (nsp + 1) / 2;
    p->deltar = deltar;
    p->dim = dim;
    // select_ncdfinput (netcdf.f90:610-617): side = minval(L(1:ndim)); rcrdf = min(rcrdf, side/2)
    float side = min_edge(box, dim);
    float half = side / 2.0f;
    float rc = fminf(rcrdf, half);
    if (!(rc > 0.f)) rc = half;  // rcrdf <= 0 means half the box (netcdf.f90:613-617)
    p->rcrdf_eff = rc;
    p->side2 = rc * rc;
    // RDF_init (rdf.cuf:55-59)
    p->lsmax = nint_host(rc / deltar) + 1;
    p->n_max = n_max;
    size_t hist_bytes = (size_t)p->nit * p->lsmax * 4;
    size_t budget = ctx->smem_optin - kSlots * kJChunk * sizeof(float4) - 4096;
    if (hist_bytes > budget) {
        delete p;
        return trj_fail(ctx, TRJ_ERR_UNSUPPORTED,
                        "rdf plan: histogram of %zu bytes exceeds shared memory (%zu); increase deltar "
                        "or reduce rcrdf", hist_bytes, budget);
    }
    cells_for(box, p->side2, p->nc, dim);
    int ncell = p->nc[0] * p->nc[1] * p->nc[2];
    // Room for a box up to 25% smaller per axis (more cells) without re-planning.
    p->ncell_cap = std::max(ncell * 2 + 64, 64);
    trj_device_guard g(ctx->device);
    // Sub-cell keys: up to 64 per cell, never more entries than atoms (or cells).
    p->fine_cap = std::max<int64_t>(p->ncell_cap, std::min<int64_t>((int64_t)p->ncell_cap * 64, n_max));
    size_t bytes = 64 + sizeof(int32_t) * (size_t)(3 * p->ncell_cap + 1) +
                   sizeof(int32_t) * (size_t)(2 * p->fine_cap + 1) +
                   (sizeof(int32_t) * 2 + sizeof(float4)) * (size_t)std::max<int64_t>(n_max, 1);
    char* base = nullptr;
    if (trj_dev_alloc(ctx, (void**)&base, bytes + 256) != cudaSuccess) {
        delete p;
        return trj_fail(ctx, TRJ_ERR_NOMEM, "rdf plan: %zu bytes of scratch", bytes);
    }
    p->sorted = reinterpret_cast<float4*>(base);
    p->akey = reinterpret_cast<int32_t*>(p->sorted + std::max<int64_t>(n_max, 1));
    p->aslot = p->akey + std::max<int64_t>(n_max, 1);
    p->ccount = p->aslot + std::max<int64_t>(n_max, 1);
    p->cstart = p->ccount + p->ncell_cap;
    p->cflag = p->cstart + p->ncell_cap + 1;
    p->fcount = p->cflag + p->ncell_cap;
    p->fstart = p->fcount + p->fine_cap;
    p->work = reinterpret_cast<unsigned long long*>(
        (reinterpret_cast<uintptr_t>(p->fstart + p->fine_cap + 1) + 15) & ~(uintptr_t)15);
    p->scratch_bytes = (int64_t)bytes;
    *out = p;
    return TRJ_OK;
}

extern "C" int trj_rdf_plan_create(trj_ctx* ctx, int nsp, float deltar, float rcrdf, const float box[3],
                                   int64_t n_max, trj_rdf_plan** out) {
    return rdf_plan_create_impl(ctx, nsp, deltar, rcrdf, box, n_max, 3, out);
}

extern "C" int trj_rdf_plan_create_2d(trj_ctx* ctx, int nsp, float deltar, float rcrdf, const float box[3],
                                      int64_t n_max, trj_rdf_plan** out) {
    return rdf_plan_create_impl(ctx, nsp, deltar, rcrdf, box, n_max, 2, out);
}

extern "C" int trj_rdf_plan_create_floor(trj_ctx* ctx, int nsp, float r_max, int nbins, const float box[3],
                                         int64_t n_max, trj_rdf_plan** out) {
    if (!ctx || !out || !box) return TRJ_ERR_INVALID;
    *out = nullptr;
    if (nbins < 1 || !(r_max > 0.f))
        return trj_fail(ctx, TRJ_ERR_INVALID, "rdf plan (floor bins): nbins=%d r_max=%g", nbins, (double)r_max);
    const float side = fminf(box[0], fminf(box[1], box[2]));
    if (!(r_max < side / 2.0f))
        return trj_fail(ctx, TRJ_ERR_INVALID, "rdf plan (floor bins): r_max=%g must be below half the box (%g)",
                        (double)r_max, (double)(side / 2.0f));
    const float deltar = r_max / (float)nbins;
    int rc = trj_rdf_plan_create(ctx, nsp, deltar, r_max, box, n_max, out);
    if (rc != TRJ_OK) return rc;
    trj_rdf_plan* p = *out;
    p->floor_bins = 1;
    p->lsmax = nbins;
    p->rcrdf_eff = r_max;
    p->side2 = r_max * r_max;
    return TRJ_OK;
}

extern "C" int trj_rdf_plan_info(const trj_rdf_plan* p, int* lsmax, int* nit, int cells[3], float* rcrdf_eff,
                                 float* side2, int64_t* scratch_bytes) {
    if (!p) return TRJ_ERR_INVALID;
    if (lsmax) *lsmax = p->lsmax;
    if (nit) *nit = p->nit;
    if (cells) for (int d = 0; d < 3; ++d) cells[d] = p->nc[d];
    if (rcrdf_eff) *rcrdf_eff = p->rcrdf_eff;
    if (side2) *side2 = p->side2;
    if (scratch_bytes) *scratch_bytes = p->scratch_bytes;
    return TRJ_OK;
}

extern "C" int trj_rdf_kernel_ms(trj_rdf_plan* p, float* ms) {
    if (!p) return TRJ_ERR_INVALID;
    return p->timer.elapsed(p->ctx, ms);
}

extern "C" int trj_rdf_plan_destroy(trj_rdf_plan* p) {
    if (!p) return TRJ_OK;
    {
        trj_device_guard g(p->ctx->device);
        trj_dev_free(p->ctx, p->sorted);
        trj_dev_free(p->ctx, p->sorted_q);
        p->timer.release();
    }
    delete p;
    return TRJ_OK;
}

// Frame accumulation; charge_dev/gqq_dev non-null adds the charge-product histogram.
static int rdf_accumulate_impl(trj_rdf_plan* plan, const float* packed_dev, const float* charge_dev, int64_t n,
                               const float box[3], uint64_t* hist_dev, uint64_t* edge_dev, double* gqq_dev,
                               void* stream) {
    if (!plan) return TRJ_ERR_INVALID;
    trj_ctx* ctx = plan->ctx;
    if (!box || !hist_dev) return trj_fail(ctx, TRJ_ERR_INVALID, "rdf accumulate: null argument");
    const bool charged = gqq_dev != nullptr;
    if (charged && n > 0 && !charge_dev)
        return trj_fail(ctx, TRJ_ERR_INVALID, "rdf accumulate: null charge array");
    if (n < 0 || n > plan->n_max)
        return trj_fail(ctx, TRJ_ERR_CAPACITY, "rdf accumulate: n=%lld exceeds plan n_max=%lld", (long long)n,
                        (long long)plan->n_max);
    if (n > 0 && (!packed_dev || ((uintptr_t)packed_dev) % 16))
        return trj_fail(ctx, TRJ_ERR_INVALID, "rdf accumulate: packed_dev null or not 16-byte aligned");
    if (!(box[0] > 0.f && box[1] > 0.f && box[2] > 0.f))
        return trj_fail(ctx, TRJ_ERR_INVALID, "rdf accumulate: box edges must be positive");
    trj_device_guard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    if (charged && !plan->sorted_q) {
        const size_t nq = (size_t)std::max<int64_t>(plan->n_max, 1);
        const size_t qbytes = ((nq * sizeof(float) + 255) & ~(size_t)255) + sizeof(double) * (size_t)plan->lsmax;
        char* qb = nullptr;
        if (trj_dev_alloc(ctx, (void**)&qb, qbytes) != cudaSuccess)
            return trj_fail(ctx, TRJ_ERR_NOMEM, "rdf accumulate: %zu bytes of charge scratch", qbytes);
        plan->sorted_q = reinterpret_cast<float*>(qb);
        plan->gqq_frame = reinterpret_cast<double*>(qb + ((nq * sizeof(float) + 255) & ~(size_t)255));
        plan->scratch_bytes += (int64_t)qbytes;
    }
    plan->cells_valid = 0;
    if (n < 2) {
        // No pair; gqq still receives 0/avq2 per bin, as the reference adds gqq_d/avq2 every frame.
        if (charged && n == 1) {
            TRJ_CUDA_TRY(ctx, cudaMemsetAsync(plan->gqq_frame, 0, sizeof(double) * plan->lsmax, s));
            gqq_finish_kernel<<<1, 1024, 0, s>>>(charge_dev, n, plan->gqq_frame, plan->lsmax, gqq_dev);
            ctx->launches += 1;
            TRJ_CUDA_TRY(ctx, cudaGetLastError());
        }
        return TRJ_OK;
    }
    // Per-frame clip, as select_ncdfinput does on every frame (netcdf.f90:610-617).
    float side = min_edge(box, plan->dim);
    plan->rcrdf_eff = fminf(plan->rcrdf_eff, side / 2.0f);
    plan->side2 = plan->rcrdf_eff * plan->rcrdf_eff;

    RdfParams P;
    memset(&P, 0, sizeof(P));
    for (int d = 0; d < 3; ++d) {
        P.L[d] = box[d];
        P.h1[d] = nint_threshold(box[d], 0.5f);
        P.h2[d] = nint_threshold(box[d], 1.5f);
    }
    P.side2 = plan->side2;
    P.side2_lo = (float)((double)plan->side2 * (1.0 - 1.0 / 1048576.0));
    P.side2_hi = (float)((double)plan->side2 * (1.0 + 1.0 / 1048576.0));
    P.deltar = plan->deltar;
    P.inv_deltar = 1.0f / plan->deltar;
    P.lsmax = plan->lsmax;
    P.floor_bins = plan->floor_bins;
    P.wait_clocks = plan->wait_clocks;
    P.stall_test = plan->stall_test;
    P.nsp = plan->nsp;
    P.nit = plan->nit;
    cells_for(box, plan->side2, P.nc, plan->dim);
    P.ncell = P.nc[0] * P.nc[1] * P.nc[2];
    if (P.ncell > plan->ncell_cap)
        return trj_fail(ctx, TRJ_ERR_CAPACITY, "rdf accumulate: %d cells exceed plan capacity %d", P.ncell,
                        plan->ncell_cap);
    for (int d = 0; d < 3; ++d) {
        plan->nc[d] = P.nc[d];
        plan->box_last[d] = box[d];
    }
    // Half-shell stencil over the split axes: (0,0,0) first, then offsets > 0 lexicographically.
    int no = 0;
    P.off[no][0] = P.off[no][1] = P.off[no][2] = 0;
    ++no;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                if ((dx && P.nc[0] == 1) || (dy && P.nc[1] == 1) || (dz && P.nc[2] == 1)) continue;
                bool pos = dx > 0 || (dx == 0 && (dy > 0 || (dy == 0 && dz > 0)));
                if (!pos) continue;
                P.off[no][0] = dx;
                P.off[no][1] = dy;
                P.off[no][2] = dz;
                ++no;
            }
    P.noff = no;
    double avg = (double)n / P.ncell;
    P.hsplit = std::max(1, (int)ceil(avg / kHomeChunk));
    // No minimum image needed away from the wrap (2D: z differences are 0, z is never wrapped).
    P.fast_ok = P.nc[0] >= 5 && P.nc[1] >= 5 && (P.nc[2] >= 5 || plan->dim == 2);
    // Cull radius 2^-10 above the cutoff (the exact test needs rr2 < side2*(1 + 2^-20)); the pad,
    // 2^-16 of the largest edge, exceeds the rounding of the box and gap arithmetic (a few ulps of
    // coordinates below 2L).
    P.cull2 = (float)((double)plan->side2 * (1.0 + 1.0 / 1024.0) * (1.0 + 1.0 / 1024.0));
    P.cull_pad = (float)((double)std::max(box[0], std::max(box[1], box[2])) / 65536.0);
    // Split neighbour ranges when there are too few (cell, offset, home chunk) items to fill the GPU.
    int64_t base_items = (int64_t)P.ncell * P.noff * P.hsplit;
    int64_t want = (int64_t)ctx->sm_count * 4;
    P.jsplit = (int)std::max<int64_t>(1, std::min<int64_t>(64, (want + base_items - 1) / base_items));
    P.nitems = base_items * P.jsplit;

    // Shared memory: two staging buffers + histogram replicas (+ FP64 charge replicas).
    size_t hist_bytes = (size_t)P.nit * P.lsmax * 4 + (charged ? (size_t)P.lsmax * 8 + 8 : 0);
    size_t stage = kSlots * kJChunk * sizeof(float4);
    size_t optin = ctx->smem_optin;
    // Most CTAs per SM (up to 4, i.e. 32 warps) that still hold >= 2 histogram replicas each;
    // a single CTA per SM otherwise.
    const size_t sm_smem = optin + 1024;  // per-SM shared memory (the opt-in limit plus the driver's block reserve)
    int ctas_per_sm = 1, nrep = 0;
    for (int k = 4; k >= 2; --k) {
        size_t per_cta = sm_smem / k - 1024 - 2048;  // driver reserve + static shared memory
        int r = per_cta > stage ? (int)std::min<size_t>(8, (per_cta - stage) / hist_bytes) : 0;
        if (r >= 2) {
            ctas_per_sm = k;
            nrep = r;
            break;
        }
    }
    if (nrep < 2) nrep = (int)std::min<size_t>(8, (optin - 2048 - stage) / hist_bytes);
    if (nrep < 1) return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "rdf accumulate: histogram too large");
    P.nrep = nrep;
    size_t smem = stage + (size_t)nrep * hist_bytes;
    void (*kern)(RdfParams, const float4*, const int32_t*, const int32_t*, const int32_t*, const int32_t*,
                 unsigned long long*, unsigned long long*, unsigned long long*, unsigned*, const float*, double*) =
        plan->floor_bins ? (charged ? rdf_pairs_kernel<true, true> : rdf_pairs_kernel<true, false>)
                         : (charged ? rdf_pairs_kernel<false, true> : rdf_pairs_kernel<false, false>);
    TRJ_CUDA_TRY(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));

    // Sub-cells per cell axis: 4 (64 per cell) from 128 atoms per cell on, 2 from 16 on, within the
    // key capacity.
    const double per_cell = (double)n / P.ncell;
    int sbits = per_cell >= 128.0 ? 2 : (per_cell >= 16.0 ? 1 : 0);
    while (sbits > 0 && ((int64_t)P.ncell << (3 * sbits)) > plan->fine_cap) --sbits;
    const int nkey = P.ncell << (3 * sbits);
    P.sbits = sbits;

    // Cell binning: count, scan over cells, sub-cell offsets, scatter.
    TRJ_CUDA_TRY(ctx, cudaMemsetAsync(plan->fcount, 0, sizeof(int32_t) * nkey, s));
    TRJ_CUDA_TRY(ctx, cudaMemsetAsync(plan->ccount, 0, sizeof(int32_t) * P.ncell, s));
    TRJ_CUDA_TRY(ctx, cudaMemsetAsync(plan->cflag, 0, sizeof(int32_t) * P.ncell, s));
    TRJ_CUDA_TRY(ctx, cudaMemsetAsync(plan->work, 0, sizeof(unsigned long long), s));
    unsigned nb = (unsigned)((n + 255) / 256);
    cell_assign_kernel<<<nb, 256, 0, s>>>((const float4*)packed_dev, n, box[0], box[1], box[2], P.nc[0],
                                          P.nc[1], P.nc[2], sbits, plan->fcount, plan->ccount, plan->cflag,
                                          plan->akey, plan->aslot);
    scan_exclusive_kernel<<<1, 1024, 0, s>>>(plan->ccount, plan->cstart, P.ncell);
    sub_offsets_kernel<<<(unsigned)((P.ncell + 7) / 8), 256, 0, s>>>(plan->fcount, plan->cstart, P.ncell, sbits,
                                                                    plan->fstart);
    cell_scatter_kernel<<<nb, 256, 0, s>>>((const float4*)packed_dev, n, plan->akey, plan->aslot, plan->fstart,
                                           plan->sorted, charged ? charge_dev : nullptr, plan->sorted_q);
    if (charged) TRJ_CUDA_TRY(ctx, cudaMemsetAsync(plan->gqq_frame, 0, sizeof(double) * plan->lsmax, s));
    int64_t grid = std::min<int64_t>((int64_t)ctx->sm_count * ctas_per_sm, P.nitems);
    plan->timer.begin(ctx, s);
    kern<<<(unsigned)grid, kThreads, smem, s>>>(P, plan->sorted, plan->cstart, plan->ccount, plan->cflag, plan->fstart,
                                                plan->work,
                                                (unsigned long long*)hist_dev, (unsigned long long*)edge_dev,
                                                ctx->status_dev, charged ? plan->sorted_q : nullptr,
                                                charged ? plan->gqq_frame : nullptr);
    plan->timer.end(ctx, s);
    plan->cells_valid = 1;
    ctx->launches += 5;
    if (charged) {
        gqq_finish_kernel<<<1, 1024, 0, s>>>(charge_dev, n, plan->gqq_frame, plan->lsmax, gqq_dev);
        ctx->launches += 1;
    }
    TRJ_CUDA_TRY(ctx, cudaGetLastError());
    return TRJ_OK;
}

extern "C" int trj_rdf_accumulate(trj_rdf_plan* plan, const float* packed_dev, int64_t n, const float box[3],
                                  uint64_t* hist_dev, uint64_t* edge_dev, void* stream) {
    return rdf_accumulate_impl(plan, packed_dev, nullptr, n, box, hist_dev, edge_dev, nullptr, stream);
}

extern "C" int trj_rdf_accumulate_charged(trj_rdf_plan* plan, const float* packed_dev, const float* charge_dev,
                                          int64_t n, const float box[3], uint64_t* hist_dev, uint64_t* edge_dev,
                                          double* gqq_dev, void* stream) {
    if (!plan) return TRJ_ERR_INVALID;
    if (!gqq_dev) return trj_fail(plan->ctx, TRJ_ERR_INVALID, "rdf accumulate (charged): null gqq");
    return rdf_accumulate_impl(plan, packed_dev, charge_dev, n, box, hist_dev, edge_dev, gqq_dev, stream);
}

extern "C" int trj_rdf_s2n(trj_rdf_plan* plan, int nrandom, uint64_t* gi_dev, uint64_t* g2i_dev, float* points_dev,
                           void* stream) {
    if (!plan) return TRJ_ERR_INVALID;
    trj_ctx* ctx = plan->ctx;
    if (nrandom < 0 || !gi_dev || !g2i_dev) return trj_fail(ctx, TRJ_ERR_INVALID, "rdf s2n: bad arguments");
    if (plan->floor_bins)
        return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "rdf s2n: needs the reference's nint bins (not a floor-bin plan)");
    if (!plan->cells_valid)
        return trj_fail(ctx, TRJ_ERR_INVALID, "rdf s2n: no frame accumulated (call trj_rdf_accumulate first)");
    if (nrandom == 0) return TRJ_OK;
    trj_device_guard g(ctx->device);
    const size_t smem = sizeof(unsigned long long) * (size_t)(plan->lsmax + 1);
    if (smem > (size_t)ctx->smem_optin - 64)
        return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "rdf s2n: lsmax=%d too large", plan->lsmax);
    if (smem > 48 * 1024)
        TRJ_CUDA_TRY(ctx, cudaFuncSetAttribute(s2n_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    s2n_kernel<<<(unsigned)nrandom, 256, smem, (cudaStream_t)stream>>>(
        plan->sorted, plan->cstart, plan->ccount, plan->box_last[0], plan->box_last[1], plan->box_last[2],
        plan->nc[0], plan->nc[1], plan->nc[2], plan->side2, plan->deltar, plan->lsmax,
        (unsigned long long*)gi_dev, (unsigned long long*)g2i_dev, points_dev, plan->dim);
    ctx->launches += 1;
    TRJ_CUDA_TRY(ctx, cudaGetLastError());
    return TRJ_OK;
}

extern "C" int trj_rdf_plan_set_binning(trj_rdf_plan* plan, int floor_bins) {
    if (!plan) return TRJ_ERR_INVALID;
    plan->floor_bins = floor_bins ? 1 : 0;
    return TRJ_OK;
}

extern "C" int trj_rdf_plan_set_wait(trj_rdf_plan* plan, int64_t clocks, int stall_test) {
    if (!plan) return TRJ_ERR_INVALID;
    if (clocks != 0 && (clocks < 1000 || clocks > TRJ_WAIT_CLOCKS))
        return trj_fail(plan->ctx, TRJ_ERR_INVALID, "trj_rdf_plan_set_wait: clocks %lld outside [1000, %lld] (0: default)",
                        (long long)clocks, (long long)TRJ_WAIT_CLOCKS);
    plan->wait_clocks = clocks ? clocks : TRJ_WAIT_CLOCKS;
    plan->stall_test = stall_test ? 1 : 0;
    return TRJ_OK;
}

// ---- fused multi-request launch: host side of the pair kernel ----------------------------------

size_t trj_batch_pairs_smem(int hist_words) { return kBatchTile * sizeof(float4) + 2 * (size_t)hist_words * 4; }

int trj_batch_pairs_prepare(int hist_words) {
    return cudaFuncSetAttribute(batch_pairs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)trj_batch_pairs_smem(hist_words)) == cudaSuccess ? 0 : -1;
}

void trj_batch_launch_pairs(BatchHeader* hdr, const BatchItem* items, const float4* packed, int hist_words,
                            int grid, cudaStream_t s) {
    batch_pairs_kernel<<<grid, kBatchThreads, trj_batch_pairs_smem(hist_words), s>>>(hdr, items, packed, hist_words);
}

int trj_batch_pairs_occupancy(int hist_words, int* per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, batch_pairs_kernel, kBatchThreads,
                                                         trj_batch_pairs_smem(hist_words)) == cudaSuccess ? 0 : -1;
}

int trj_batch_fill_rdf(trj_rdf_plan* plan, const float box[3], int hist_words, BatchItem* it, int* nsp) {
    trj_ctx* ctx = plan->ctx;
    if (plan->dim != 3) return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "batch: two-dimensional pair plans run unfused");
    if (plan->nsp > kBatchMaxSpecies)
        return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "batch: %d species (1..%d)", plan->nsp, kBatchMaxSpecies);
    if ((int64_t)plan->nit * plan->lsmax > hist_words)
        return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "batch: a histogram of %d x %d bins exceeds the batch's %d words",
                        plan->nit, plan->lsmax, hist_words);
    // the per-frame clip of trj_rdf_accumulate (netcdf.f90:610-617)
    const float side = min_edge(box, plan->dim);
    plan->rcrdf_eff = fminf(plan->rcrdf_eff, side / 2.0f);
    plan->side2 = plan->rcrdf_eff * plan->rcrdf_eff;
    plan->cells_valid = 0;
    for (int d = 0; d < 3; ++d) {
        it->h1[d] = nint_threshold(box[d], 0.5f);
        it->h2[d] = nint_threshold(box[d], 1.5f);
    }
    it->side2 = plan->side2;
    it->side2_lo = (float)((double)plan->side2 * (1.0 - 1.0 / 1048576.0));
    it->side2_hi = (float)((double)plan->side2 * (1.0 + 1.0 / 1048576.0));
    it->deltar = plan->deltar;
    it->inv_deltar = 1.0f / plan->deltar;
    it->lsmax = plan->lsmax;
    it->nit = plan->nit;
    it->floor_bins = plan->floor_bins;
    *nsp = plan->nsp;
    return TRJ_OK;
}
