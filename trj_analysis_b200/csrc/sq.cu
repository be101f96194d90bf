// sq.cu -- S_ab(Q) plan, direct-sum kernel, and the FP64 shell reduction.
//
// rho_a(k) = sum_{j in species a} exp(i k.r_j) for lattice vectors k = 2*pi*(nx/Lx, ny/Ly, nz/Lz).
// The phase of every term is reduced exactly: each coordinate becomes the 32-bit fixed-point
// fraction u = (x/L mod 1) * 2^32 (computed in FP64, once per atom and frame), and
// n.u mod 2^32 is evaluated in wrapping integer arithmetic, so the angle handed to the FP32
// sine/cosine is always in [-pi, pi).  The reference (src/modules/sq.cuf:537-581, sqfnD)
// forms x*kf1 + y*kf2 + z*kf3 in FP32 and calls __cosf/__sinf on arguments up to ~L*q; the
// exact reduction keeps the per-term error at the FP32 level instead.
//
// Output per bin b and species pair (a<=b'): sum_{k in b} w_k Re(rho_a(k) conj(rho_b'(k))),
// accumulated in FP64 with a fixed reduction order (one CTA per bin), so results do not depend
// on scheduling.  The reference's sqfp (self partials) and sqf (bsc-weighted total,
// sq.cuf:583-588) are linear combinations of these rows.
#include <math.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "batch.cuh"
#include "sq_plan.cuh"

namespace {

constexpr int kPlainThreads = 256;
constexpr int kPlainVPT = 4;           // k-vectors per thread
constexpr int kPlainChunk = 1024;      // atoms staged per pass
constexpr int kPlainSub = 64;          // FP32 partial-sum length before the FP64 add

// Fixed-point phase coordinates of every atom.  With charges (q non-null) every atom is written a
// second time at n + i as a member of the charge species qsp, its charge (FP32 bits) in place of the
// species index: rho_q(k) = sum_j q_j exp(i k.r_j) (sq.cuf:569-573) is then the sum of that species.
// zmul != 0 (planar frames in tile form): the third phase is zmul * u_y mod 2^32, exactly, so that
// lattice vector (nx, ny mod zmul, ny div zmul) has the phase of (nx, ny) in the plane.
__global__ void phase_coords_kernel(const float4* __restrict__ packed, int64_t n, double Lx, double Ly,
                                    double Lz, uint4* __restrict__ out, const float* __restrict__ q,
                                    unsigned zmul) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = packed[i];
    unsigned u[3] = {trj_phase_fraction(v.x, Lx), trj_phase_fraction(v.y, Ly), trj_phase_fraction(v.z, Lz)};
    if (zmul) u[2] = u[1] * zmul;
    out[i] = make_uint4(u[0], u[1], u[2], (unsigned)__float_as_int(v.w));
    if (q) out[n + i] = make_uint4(u[0], u[1], u[2], __float_as_uint(q[i]));
}

// cos and sin of the angle 2 pi ph / 2^32 (ph a 32-bit fixed-point fraction of a turn): the nearest of
// 256 table angles (the table holds cos, sin of 2 pi k / 256, each rounded once from FP64), rotated by the
// remainder |theta| <= pi/256 through its Taylor polynomials (theta - theta^3/6; 1 - theta^2/2 +
// theta^4/24, truncation below 3e-12).  Every step rounds to nearest once, so the error has no
// systematic part, which matters because it is added once per atom.
__device__ __forceinline__ void sincos_turn(unsigned ph, const float2* __restrict__ tab, float& sn, float& cs) {
    const unsigned hi = (ph + 0x800000u) >> 24;         // nearest table angle (mod 256)
    const int lo = (int)(ph - (hi << 24));               // remainder in [-2^23, 2^23): exact as a float
    const float th = (float)lo * 1.4629180792671596e-09f;  // 2 pi / 2^32
    const float t2 = th * th;
    const float sl = th * fmaf(t2, -0.16666667f, 1.0f);
    const float cl = fmaf(t2, fmaf(t2, 0.041666668f, -0.5f), 1.0f);
    const float2 t = tab[hi & 255u];
    cs = fmaf(t.x, cl, -(t.y * sl));
    sn = fmaf(t.y, cl, t.x * sl);
}

// cos, sin(2 pi k / 256), k = 0..255, each rounded once from FP64 (the table of sincos_turn).
__device__ __forceinline__ void fill_turn_table(float2* turn_tab) {
    for (int k = threadIdx.x; k < 256; k += blockDim.x) {
        double sd, cd;
        sincospi((double)k / 128.0, &sd, &cd);
        turn_tab[k] = make_float2((float)cd, (float)sd);
    }
}

// Direct sum of one block of vectors (bx) over one slice (by of nsplit) of every species: thread owns
// VPT vectors.  Species qsp (if any) is the charge species: each term is weighted by the charge in the
// entry's w.  Partials by position in the subset: part[by][species][nsub].  turn_tab must be filled
// (fill_turn_table) before the call; the barrier at the top of the chunk loop orders it.
template <int VPT>
__device__ __forceinline__ void plain_block(const uint4* __restrict__ phase, const int64_t* __restrict__ sp_off,
                                            int nsp, int qsp, const int4* __restrict__ vecs,
                                            const int32_t* __restrict__ subset, int nsub, int nsplit,
                                            double2* __restrict__ part, int64_t bx, int64_t by, uint4* atoms,
                                            const float2* turn_tab) {
    const int tid = threadIdx.x;
    const int64_t vbase = bx * kPlainThreads * VPT;
    unsigned nx[VPT], ny[VPT], nz[VPT];
    int vidx[VPT];
#pragma unroll
    for (int q = 0; q < VPT; ++q) {
        int64_t s = vbase + q * kPlainThreads + tid;
        vidx[q] = s < nsub ? subset[s] : -1;
        int4 v = vidx[q] >= 0 ? vecs[vidx[q]] : make_int4(0, 0, 0, 0);
        nx[q] = (unsigned)v.x;
        ny[q] = (unsigned)v.y;
        nz[q] = (unsigned)v.z;
    }
    for (int a = 0; a < nsp; ++a) {
        int64_t a0 = sp_off[a], a1 = sp_off[a + 1];
        int64_t len = a1 - a0;
        int64_t s0 = a0 + len * by / nsplit, s1 = a0 + len * (by + 1) / nsplit;
        double accr[VPT], acci[VPT];
#pragma unroll
        for (int q = 0; q < VPT; ++q) accr[q] = acci[q] = 0.0;
        const bool weighted = a == qsp;
        for (int64_t c0 = s0; c0 < s1; c0 += kPlainChunk) {
            int cnt = (int)((s1 - c0) < (int64_t)kPlainChunk ? (s1 - c0) : (int64_t)kPlainChunk);
            __syncthreads();
            for (int k = tid; k < cnt; k += kPlainThreads) atoms[k] = phase[c0 + k];
            __syncthreads();
            for (int j0 = 0; j0 < cnt; j0 += kPlainSub) {
                int j1 = min(cnt, j0 + kPlainSub);
                float fr[VPT], fi[VPT];
#pragma unroll
                for (int q = 0; q < VPT; ++q) fr[q] = fi[q] = 0.f;
                for (int j = j0; j < j1; ++j) {
                    uint4 u = atoms[j];
                    const float w = weighted ? __uint_as_float(u.w) : 1.0f;  // fma with 1: the plain sum
#pragma unroll
                    for (int q = 0; q < VPT; ++q) {
                        unsigned ph = nx[q] * u.x + ny[q] * u.y + nz[q] * u.z;
                        // an unbiased sine/cosine: a biased fast one adds its mean error once per
                        // atom, which at 10^6 atoms is a few 1e-5 of |rho|^2 on a shell of three vectors
                        float sn, cs;
                        sincos_turn(ph, turn_tab, sn, cs);
                        fr[q] = fmaf(w, cs, fr[q]);
                        fi[q] = fmaf(w, sn, fi[q]);
                    }
                }
#pragma unroll
                for (int q = 0; q < VPT; ++q) {
                    accr[q] += (double)fr[q];
                    acci[q] += (double)fi[q];
                }
            }
        }
#pragma unroll
        for (int q = 0; q < VPT; ++q)
            if (vidx[q] >= 0)  // partials by position in the subset: [split][species][nsub]
                part[(by * nsp + a) * nsub + vbase + q * kPlainThreads + tid] = make_double2(accr[q], acci[q]);
    }
}

template <int VPT>
__global__ void __launch_bounds__(kPlainThreads) sq_plain_kernel(
    const uint4* __restrict__ phase, const int64_t* __restrict__ sp_off, int nsp, int qsp,
    const int4* __restrict__ vecs, const int32_t* __restrict__ subset, int nsub, int64_t nvec,
    int nsplit, double2* __restrict__ part) {
    __shared__ uint4 atoms[kPlainChunk];
    __shared__ float2 turn_tab[256];
    fill_turn_table(turn_tab);
    plain_block<VPT>(phase, sp_off, nsp, qsp, vecs, subset, nsub, nsplit, part, blockIdx.x, blockIdx.y, atoms,
                     turn_tab);
}

// rho[a][v] = sum over splits (fixed order) for the subset's vectors.
__global__ void gather_plain_kernel(const double2* __restrict__ part, const int32_t* __restrict__ subset,
                                    int nsub, int64_t nvec, int nsp, int nsplit, double2* __restrict__ rho) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)nsub * nsp) return;
    int a = (int)(t / nsub);
    const int64_t pos = t % nsub;
    int v = subset[pos];
    double re = 0.0, im = 0.0;
    for (int s = 0; s < nsplit; ++s) {
        double2 p = part[((int64_t)s * nsp + a) * nsub + pos];
        re += p.x;
        im += p.y;
    }
    rho[(int64_t)a * nvec + v] = make_double2(re, im);
}

// rho[a][v] for tensor-tile vectors from the FP64 tile blocks.
__global__ void gather_dense_kernel(const double* __restrict__ tc_out, const int64_t* __restrict__ src,
                                    int64_t nvec, int nsp, const int64_t* __restrict__ tile_species_stride,
                                    double2* __restrict__ rho) {
    int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvec) return;
    int64_t o = src[v];
    if (o < 0) return;
    int64_t stride = tile_species_stride[v];
    const bool conj = stride < 0;  // evaluated through -k: rho(k) = conj(rho(-k))
    if (conj) stride = -stride;
    for (int a = 0; a < nsp; ++a) {
        const double* b = tc_out + o + a * stride;
        rho[(int64_t)a * nvec + v] = make_double2(b[0], conj ? -b[kTcRows] : b[kTcRows]);
    }
}

// out[bin][pair] += sum_v w_v Re(rho_a conj(rho_b)) over the bin's vectors [v0, v1), by one CTA of
// 256 threads in a fixed order (thread-strided FP64 sums, warp shuffles, warps in order).
__device__ __forceinline__ void bin_reduce_block(const double2* __restrict__ rho, const double* __restrict__ w,
                                                 int v0, int v1, int64_t nvec, int nsp, int bin,
                                                 double* __restrict__ out, double* red) {
    const int nit = nsp * (nsp + 1) / 2;
    for (int a = 0; a < nsp; ++a)
        for (int b = a; b < nsp; ++b) {
            double s = 0.0;
            for (int v = v0 + threadIdx.x; v < v1; v += blockDim.x) {
                double2 ra = rho[(int64_t)a * nvec + v], rb = rho[(int64_t)b * nvec + v];
                s += w[v] * (ra.x * rb.x + ra.y * rb.y);
            }
            for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
            __syncthreads();
            if (threadIdx.x == 0) {
                double t = 0.0;
                for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
                out[(int64_t)bin * nit + trj_pair_row(a, b, nsp)] += t;
            }
            __syncthreads();
        }
}

// One CTA per bin.
__global__ void bin_reduce_kernel(const double2* __restrict__ rho, const double* __restrict__ w,
                                  const int32_t* __restrict__ bin_start, int64_t nvec, int nsp,
                                  double* __restrict__ out) {
    __shared__ double red[32];
    const int bin = blockIdx.x;
    const int v0 = bin_start[bin], v1 = bin_start[bin + 1];
    if (v0 >= v1) return;
    bin_reduce_block(rho, w, v0, v1, nvec, nsp, bin, out, red);
}

// ---- fused multi-request launch: direct sum and shell reduction of every packed frame ----------
//
// The same blocks as sq_plain_kernel and gather_plain_kernel + bin_reduce_kernel with each item's own
// plan, vector blocks and splits, so an item's sums are bit-identical to the single-request plain
// method.  Units come from global counters: (item, vector block, split) for the direct sum, (item,
// bin) for the reduction.
__global__ void __launch_bounds__(kPlainThreads, 2) batch_sq_kernel(BatchHeader* __restrict__ hdr,
                                                                    const BatchItem* __restrict__ items,
                                                                    const uint4* __restrict__ phase) {
    __shared__ uint4 atoms[kPlainChunk];
    __shared__ float2 turn_tab[256];
    __shared__ long long unit_s;
    fill_turn_table(turn_tab);
    const int nitems = hdr->nitems;
    const int64_t total = hdr->total_sq;
    while (true) {
        if (threadIdx.x == 0) unit_s = (long long)atomicAdd(&hdr->counter[1], 1ull);
        __syncthreads();
        const int64_t u = unit_s;
        __syncthreads();
        if (u >= total) break;
        const BatchItem& it = items[batch_item_of<&BatchItem::sq_begin>(items, nitems, u)];
        const int64_t t = u - it.sq_begin, bx = t % it.nvblk, by = t / it.nvblk;
        if (it.vpt == 1)
            plain_block<1>(phase + it.atom_off, it.sp_off_dev, it.nsp, -1, it.vecs, it.subset, it.nvec, it.nsplit,
                           it.part, bx, by, atoms, turn_tab);
        else
            plain_block<kPlainVPT>(phase + it.atom_off, it.sp_off_dev, it.nsp, -1, it.vecs, it.subset, it.nvec,
                                   it.nsplit, it.part, bx, by, atoms, turn_tab);
    }
}

__global__ void __launch_bounds__(256, 2) batch_reduce_kernel(BatchHeader* __restrict__ hdr,
                                                           const BatchItem* __restrict__ items) {
    __shared__ double red[32];
    __shared__ long long unit_s;
    const int nitems = hdr->nitems;
    const int64_t total = hdr->total_red;
    while (true) {
        if (threadIdx.x == 0) unit_s = (long long)atomicAdd(&hdr->counter[2], 1ull);
        __syncthreads();
        const int64_t u = unit_s;
        __syncthreads();
        if (u >= total) break;
        const BatchItem& it = items[batch_item_of<&BatchItem::red_begin>(items, nitems, u)];
        const int bin = (int)(u - it.red_begin);
        const int v0 = it.bin_start[bin], v1 = it.bin_start[bin + 1];
        if (v0 >= v1) continue;  // block-uniform
        // rho of the bin's vectors: the splits' partials in order (gather_plain_kernel; the subset is
        // every vector, so position = vector)
        const int nb = v1 - v0, nsp = it.nsp, nvec = it.nvec;
        for (int q = threadIdx.x; q < nb * nsp; q += blockDim.x) {
            const int a = q / nb, v = v0 + q % nb;
            double re = 0.0, im = 0.0;
            for (int s = 0; s < it.nsplit; ++s) {
                const double2 p = it.part[((int64_t)s * nsp + a) * nvec + v];
                re += p.x;
                im += p.y;
            }
            it.rho[(int64_t)a * nvec + v] = make_double2(re, im);
        }
        __syncthreads();
        bin_reduce_block(it.rho, it.w, v0, v1, nvec, nsp, bin, it.out, red);
    }
}

__global__ void unpermute_rho_kernel(const double2* __restrict__ rho, const int4* __restrict__ vecs,
                                     int64_t nvec, int nsp, double2* __restrict__ out) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nvec * nsp) return;
    int64_t a = t / nvec, v = t % nvec;
    out[a * nvec + vecs[v].w] = rho[t];
}

__global__ void check_counts_kernel(const uint4* __restrict__ phase, const int64_t* __restrict__ sp_off, int nsp,
                                    int64_t n, unsigned* status) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int s = (int)phase[i].w;
    if (s < 0 || s >= nsp || i < sp_off[s] || i >= sp_off[s + 1]) trj_raise(status, TRJ_DEV_COUNT_MISMATCH);
}

// Vectors per thread: 4 for large vector sets; 1 when 4 per thread would leave most lanes idle
// (the few hundred axis vectors next to the tensor tiles).
int plain_vpt(int64_t nsub) { return nsub < (int64_t)kPlainThreads * kPlainVPT * 32 ? 1 : kPlainVPT; }

int plain_nsplit(const trj_ctx* ctx, int64_t nsub, int64_t n_total) {
    const int vpt = plain_vpt(nsub);
    int64_t blocks_v = (nsub + kPlainThreads * vpt - 1) / (kPlainThreads * vpt);
    if (blocks_v <= 0) return 1;
    int64_t target = (int64_t)ctx->sm_count * 8;
    int64_t ns = (target + blocks_v - 1) / blocks_v;
    int64_t by_atoms = std::max<int64_t>(1, n_total / (2 * kPlainChunk));
    ns = std::min<int64_t>(ns, by_atoms);
    // partials are nsplit x species x vectors x 16 bytes: allow more splits for small vector sets
    const int64_t cap = nsub <= 32768 ? 1024 : 128;
    ns = std::max<int64_t>(1, std::min<int64_t>(ns, cap));
    return (int)ns;
}

}  // namespace

static void sq_plan_free(trj_sq_plan* p) {
    trj_device_guard g(p->ctx->device);
    void* ptrs[] = {p->vec_dev, p->weight_dev, p->bin_start_dev, p->species_off_dev, p->plain_all_dev,
                    p->plain_sparse_dev, p->tiles_dev, p->dense_src_dev, p->phase_dev, p->part_dev,
                    p->tc_out_dev, p->rho_dev};
    for (void* q : ptrs) trj_dev_free(p->ctx, q);
    trj_sq_tc_release(p);
    trj_dev_free(p->ctx, p->groups_buf);
    p->timer.release();
}

extern "C" int trj_sq_plan_destroy(trj_sq_plan* p) {
    if (!p) return TRJ_OK;
    sq_plan_free(p);
    delete p;
    return TRJ_OK;
}

template <class T>
static int dev_upload(trj_ctx* ctx, T** dst, const T* src, size_t count, int64_t* acct) {
    size_t bytes = std::max<size_t>(1, count) * sizeof(T);
    if (trj_dev_alloc(ctx, (void**)dst, bytes) != cudaSuccess)
        return trj_fail(ctx, TRJ_ERR_NOMEM, "sq plan: %zu bytes", bytes);
    *acct += (int64_t)bytes;
    if (count && src && cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
        return trj_fail(ctx, TRJ_ERR_CUDA, "sq plan: upload failed");
    return TRJ_OK;
}

extern "C" int trj_sq_plan_create(trj_ctx* ctx, int nsp, int64_t nvec, const int32_t* vec_host,
                                  const int32_t* bin_host, const double* weight_host, const uint8_t* dense_host,
                                  int nbins, const int64_t* species_counts, trj_sq_plan** out) {
    if (!ctx || !out) return TRJ_ERR_INVALID;
    *out = nullptr;
    if (nsp < 1 || nsp > 16) return trj_fail(ctx, TRJ_ERR_INVALID, "sq plan: nsp=%d (1..16)", nsp);
    if (nvec < 0 || nvec > (int64_t)INT32_MAX / 2 || nbins < 1)
        return trj_fail(ctx, TRJ_ERR_INVALID, "sq plan: nvec=%lld nbins=%d", (long long)nvec, nbins);
    if (nvec > 0 && (!vec_host || !bin_host || !weight_host))
        return trj_fail(ctx, TRJ_ERR_INVALID, "sq plan: null vector arrays");
    if (!species_counts) return trj_fail(ctx, TRJ_ERR_INVALID, "sq plan: null species counts");
    for (int64_t v = 0; v < nvec; ++v)
        if (bin_host[v] < 0 || bin_host[v] >= nbins)
            return trj_fail(ctx, TRJ_ERR_INVALID, "sq plan: vector %lld has bin %d outside 0..%d", (long long)v,
                            bin_host[v], nbins - 1);
    trj_sq_plan* p = new trj_sq_plan();
    p->ctx = ctx;
    p->nsp = nsp;
    p->nit = nsp * (nsp + 1) / 2;
    p->nbins = nbins;
    p->nvec = nvec;
    p->species_counts.assign(species_counts, species_counts + nsp);
    p->species_off.assign(nsp + 1, 0);
    for (int a = 0; a < nsp; ++a) {
        if (species_counts[a] < 0) {
            delete p;
            return trj_fail(ctx, TRJ_ERR_INVALID, "sq plan: negative species count");
        }
        p->species_off[a + 1] = p->species_off[a] + species_counts[a];
    }
    p->n_total = p->species_off[nsp];
    p->n_atoms = p->n_total;
    // Plan order: stable sort by bin.
    std::vector<int64_t> order(nvec);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return bin_host[x] < bin_host[y]; });
    std::vector<int4> vecs(nvec);
    std::vector<double> w(nvec);
    std::vector<int32_t> bstart(nbins + 1, 0);
    std::vector<int32_t> all(nvec), sparse;
    std::vector<int64_t> dense_idx;
    for (int64_t k = 0; k < nvec; ++k) {
        int64_t c = order[k];
        vecs[k] = make_int4(vec_host[3 * c], vec_host[3 * c + 1], vec_host[3 * c + 2], (int)c);
        w[k] = weight_host[c];
        bstart[bin_host[c] + 1] += 1;
        all[k] = (int32_t)k;
        if (dense_host && dense_host[c]) dense_idx.push_back(k);
        else sparse.push_back((int32_t)k);
    }
    for (int b = 0; b < nbins; ++b) bstart[b + 1] += bstart[b];

    // Tensor tiles over the dense vectors.  rho(-k) = conj(rho(k)), so every vector is evaluated
    // through its representative with (nx, ny) in the half plane {ny > 0, or ny == 0 and nx >= 0}
    // (the negated vector, conjugated, when its own (nx, ny) is outside).  Representatives are
    // grouped by (nx/16, ny/8) blocks; a block's nz span (both signs) becomes the tile's columns,
    // split into column groups of <= 224 (112 nz values).  A negative stride marks a conjugate.
    std::vector<int64_t> dense_src(nvec, -1), dense_stride(nvec, 0);
    const int max_cols = ctx->sq_tile_cols > 0 ? ctx->sq_tile_cols : kTcMaxCols;  // a multiple of 16
    if (!dense_idx.empty()) {
        struct Rep { int x, y, z; bool conj; };
        std::vector<Rep> rep(nvec);
        std::vector<std::pair<std::pair<int, int>, int64_t>> keyed;
        keyed.reserve(dense_idx.size());
        auto fdiv = [](int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); };
        for (int64_t k : dense_idx) {
            const int x = vecs[k].x, y = vecs[k].y, z = vecs[k].z;
            const bool in_half = y > 0 || (y == 0 && x >= 0);
            rep[k] = in_half ? Rep{x, y, z, false} : Rep{-x, -y, -z, true};
            keyed.push_back({{fdiv(rep[k].x, kTcTileNx), fdiv(rep[k].y, kTcTileNy)}, k});
        }
        std::sort(keyed.begin(), keyed.end(), [&](const auto& A, const auto& B) {
            if (A.first != B.first) return A.first < B.first;
            return rep[A.second].z < rep[B.second].z;
        });
        int64_t off = 0;
        size_t i = 0;
        while (i < keyed.size()) {
            size_t j = i;
            while (j < keyed.size() && keyed[j].first == keyed[i].first) ++j;
            // nz values of this block, sorted ascending in keyed[i..j)
            size_t a = i;
            while (a < j) {
                int z0 = rep[keyed[a].second].z;
                size_t b = a;
                while (b < j && rep[keyed[b].second].z - z0 < max_cols / 2) ++b;
                int zspan = rep[keyed[b - 1].second].z - z0 + 1;
                int ncols = ((2 * zspan + 15) / 16) * 16;
                SqTile t;
                t.nx0 = keyed[a].first.first * kTcTileNx;
                t.ny0 = keyed[a].first.second * kTcTileNy;
                t.nz0 = z0;
                t.ncols = ncols;
                t.out_off = off;
                for (size_t q = a; q < b; ++q) {
                    int64_t k = keyed[q].second;
                    int row = (rep[k].x - t.nx0) + kTcTileNx * (rep[k].y - t.ny0);
                    int col = 2 * (rep[k].z - t.nz0);
                    dense_src[k] = off + (int64_t)col * kTcRows + row;
                    dense_stride[k] = (rep[k].conj ? -1 : 1) * (int64_t)ncols * kTcRows;
                }
                p->tile_slots += (int64_t)kTcRows * (ncols / 2);
                off += (int64_t)nsp * ncols * kTcRows;
                p->tiles.push_back(t);
                a = b;
            }
            i = j;
        }
        p->tc_out_doubles = off;
        p->n_dense = (int64_t)dense_idx.size();
    }
    p->n_sparse = (int64_t)sparse.size();

    trj_device_guard g(ctx->device);
    int64_t acct = 0;
    int rc = TRJ_OK;
    std::vector<int64_t> sp_off = p->species_off;
    if ((rc = dev_upload(ctx, &p->vec_dev, vecs.data(), vecs.size(), &acct)) ||
        (rc = dev_upload(ctx, &p->weight_dev, w.data(), w.size(), &acct)) ||
        (rc = dev_upload(ctx, &p->bin_start_dev, bstart.data(), bstart.size(), &acct)) ||
        (rc = dev_upload(ctx, &p->species_off_dev, sp_off.data(), sp_off.size(), &acct)) ||
        (rc = dev_upload(ctx, &p->plain_all_dev, all.data(), all.size(), &acct)) ||
        (rc = dev_upload(ctx, &p->plain_sparse_dev, sparse.data(), sparse.size(), &acct))) {
        sq_plan_free(p);
        delete p;
        return rc;
    }
    if (!p->tiles.empty()) {
        // dense_src and per-vector species stride packed side by side
        std::vector<int64_t> both(2 * nvec);
        for (int64_t k = 0; k < nvec; ++k) {
            both[k] = dense_src[k];
            both[nvec + k] = dense_stride[k];
        }
        if ((rc = dev_upload(ctx, &p->dense_src_dev, both.data(), both.size(), &acct)) ||
            (rc = dev_upload(ctx, &p->tiles_dev, p->tiles.data(), p->tiles.size(), &acct))) {
            sq_plan_free(p);
            delete p;
            return rc;
        }
        size_t tb = sizeof(double) * (size_t)p->tc_out_doubles;
        if (trj_dev_alloc(ctx, (void**)&p->tc_out_dev, tb) != cudaSuccess) {
            sq_plan_free(p);
            delete p;
            return trj_fail(ctx, TRJ_ERR_NOMEM, "sq plan: tensor output %zu bytes", tb);
        }
        acct += (int64_t)tb;
    }
    p->nsplit_all = plain_nsplit(ctx, nvec, p->n_total);
    p->nsplit_sparse = plain_nsplit(ctx, p->n_sparse, p->n_total);
    size_t phase_b = sizeof(uint4) * (size_t)std::max<int64_t>(1, p->n_total);
    size_t part_b = sizeof(double2) * (size_t)nsp *
                    std::max<size_t>((size_t)p->nsplit_all * std::max<int64_t>(1, nvec),
                                     (size_t)p->nsplit_sparse * std::max<int64_t>(1, p->n_sparse));
    size_t rho_b = sizeof(double2) * (size_t)nsp * (size_t)std::max<int64_t>(1, nvec);
    if (trj_dev_alloc(ctx, (void**)&p->phase_dev, phase_b) != cudaSuccess ||
        trj_dev_alloc(ctx, (void**)&p->part_dev, part_b) != cudaSuccess ||
        trj_dev_alloc(ctx, (void**)&p->rho_dev, rho_b) != cudaSuccess) {
        sq_plan_free(p);
        delete p;
        return trj_fail(ctx, TRJ_ERR_NOMEM, "sq plan: scratch allocation failed");
    }
    acct += (int64_t)(phase_b + part_b + rho_b);
    p->scratch_bytes = acct;
    if (!p->tiles.empty()) {
        rc = trj_sq_tc_prepare(p);
        if (rc != TRJ_OK && rc != TRJ_ERR_UNSUPPORTED) {
            sq_plan_free(p);
            delete p;
            return rc;
        }
    }
    *out = p;
    return TRJ_OK;
}

extern "C" int trj_sq_plan_create_charged(trj_ctx* ctx, int nsp, int64_t nvec, const int32_t* vec_host,
                                          const int32_t* bin_host, const double* weight_host,
                                          const uint8_t* dense_host, int nbins, const int64_t* species_counts,
                                          trj_sq_plan** out) {
    if (!ctx || !out) return TRJ_ERR_INVALID;
    *out = nullptr;
    if (nsp < 1 || nsp > 15) return trj_fail(ctx, TRJ_ERR_INVALID, "sq plan (charged): nsp=%d (1..15)", nsp);
    if (!species_counts) return trj_fail(ctx, TRJ_ERR_INVALID, "sq plan: null species counts");
    // species nsp is the charge density over every atom
    std::vector<int64_t> counts(species_counts, species_counts + nsp);
    int64_t total = 0;
    for (int64_t c : counts) total += c;
    counts.push_back(total);
    int rc = trj_sq_plan_create(ctx, nsp + 1, nvec, vec_host, bin_host, weight_host, dense_host, nbins,
                                counts.data(), out);
    if (rc != TRJ_OK) return rc;
    (*out)->qsp = nsp;
    (*out)->n_atoms = total;
    return TRJ_OK;
}

extern "C" int trj_sq_plan_info(const trj_sq_plan* p, int64_t* n_dense, int64_t* n_tiles, int64_t* tile_slots,
                                int64_t* scratch_bytes) {
    if (!p) return TRJ_ERR_INVALID;
    if (n_dense) *n_dense = p->n_dense;
    if (n_tiles) *n_tiles = (int64_t)p->tiles.size();
    if (tile_slots) *tile_slots = p->tile_slots;
    if (scratch_bytes) *scratch_bytes = p->scratch_bytes;
    return TRJ_OK;
}

static int run_plain(trj_sq_plan* p, const int32_t* subset, int64_t nsub, int nsplit, cudaStream_t s,
                     bool timed) {
    if (nsub <= 0) return TRJ_OK;
    const int vpt = plain_vpt(nsub);
    dim3 grid((unsigned)((nsub + kPlainThreads * vpt - 1) / (kPlainThreads * vpt)), (unsigned)nsplit);
    if (timed) p->timer.begin(p->ctx, s);
    if (vpt == 1)
        sq_plain_kernel<1><<<grid, kPlainThreads, 0, s>>>(p->phase_dev, p->species_off_dev, p->nsp, p->qsp, p->vec_dev,
                                                          subset, (int)nsub, p->nvec, nsplit, p->part_dev);
    else
        sq_plain_kernel<kPlainVPT><<<grid, kPlainThreads, 0, s>>>(p->phase_dev, p->species_off_dev, p->nsp, p->qsp,
                                                                  p->vec_dev, subset, (int)nsub, p->nvec, nsplit,
                                                                  p->part_dev);
    if (timed) p->timer.end(p->ctx, s);
    int64_t tot = nsub * p->nsp;
    gather_plain_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(p->part_dev, subset, (int)nsub, p->nvec,
                                                                      p->nsp, nsplit, p->rho_dev);
    p->ctx->launches += 2;
    return TRJ_OK;
}

static int sq_accumulate_impl(trj_sq_plan* p, const float* packed_dev, const float* charge_dev, int64_t n,
                              const float box[3], int method, double* out_dev, void* stream) {
    trj_ctx* ctx = p->ctx;
    if (!box || !out_dev) return trj_fail(ctx, TRJ_ERR_INVALID, "sq accumulate: null argument");
    if (n != p->n_atoms)
        return trj_fail(ctx, TRJ_ERR_INVALID, "sq accumulate: n=%lld but the plan's species counts sum to %lld",
                        (long long)n, (long long)p->n_atoms);
    if (n > 0 && (!packed_dev || ((uintptr_t)packed_dev) % 16))
        return trj_fail(ctx, TRJ_ERR_INVALID, "sq accumulate: packed_dev null or not 16-byte aligned");
    if (!(box[0] > 0.f && box[1] > 0.f && box[2] > 0.f))
        return trj_fail(ctx, TRJ_ERR_INVALID, "sq accumulate: box edges must be positive");
    if (method != TRJ_SQ_PLAIN_FP32 && method != TRJ_SQ_SPLIT_BF16X3)
        return trj_fail(ctx, TRJ_ERR_INVALID, "sq accumulate: unknown method %d", method);
    if (p->nvec == 0) return TRJ_OK;
    trj_device_guard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    if (n > 0) {
        phase_coords_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>((const float4*)packed_dev, n, (double)box[0],
                                                                       (double)box[1], (double)box[2], p->phase_dev,
                                                                       charge_dev, p->z_from_y);
        // the charge entries (n .. 2n-1) are the same atoms: only the first n carry species to check
        check_counts_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p->phase_dev, p->species_off_dev,
                                                                        p->qsp >= 0 ? p->qsp : p->nsp, n,
                                                                        ctx->status_dev);
        ctx->launches += 2;
    }
    if (method == TRJ_SQ_PLAIN_FP32 || p->tiles.empty()) {
        run_plain(p, p->plain_all_dev, p->nvec, p->nsplit_all, s, true);
    } else {
        int rc = trj_sq_tc_run(p, box, s);
        if (rc != TRJ_OK) return rc;
        gather_dense_kernel<<<(unsigned)((p->nvec + 255) / 256), 256, 0, s>>>(
            p->tc_out_dev, p->dense_src_dev, p->nvec, p->nsp, p->dense_src_dev + p->nvec, p->rho_dev);
        ctx->launches += 1;
        run_plain(p, p->plain_sparse_dev, p->n_sparse, p->nsplit_sparse, s, false);
    }
    bin_reduce_kernel<<<p->nbins, 256, 0, s>>>(p->rho_dev, p->weight_dev, p->bin_start_dev, p->nvec, p->nsp,
                                              out_dev);
    ctx->launches += 1;
    p->last_method = method;
    TRJ_CUDA_TRY(ctx, cudaGetLastError());
    return TRJ_OK;
}

extern "C" int trj_sq_accumulate(trj_sq_plan* p, const float* packed_dev, int64_t n, const float box[3], int method,
                                 double* out_dev, void* stream) {
    if (!p) return TRJ_ERR_INVALID;
    if (p->qsp >= 0)
        return trj_fail(p->ctx, TRJ_ERR_INVALID, "sq accumulate: plan made for charges; use trj_sq_accumulate_charged");
    return sq_accumulate_impl(p, packed_dev, nullptr, n, box, method, out_dev, stream);
}

extern "C" int trj_sq_accumulate_charged(trj_sq_plan* p, const float* packed_dev, const float* charge_packed_dev,
                                         int64_t n, const float box[3], int method, double* out_dev, void* stream) {
    if (!p) return TRJ_ERR_INVALID;
    if (p->qsp < 0)
        return trj_fail(p->ctx, TRJ_ERR_INVALID, "sq accumulate (charged): plan made without charges");
    if (n > 0 && !charge_packed_dev)
        return trj_fail(p->ctx, TRJ_ERR_INVALID, "sq accumulate (charged): null charge array");
    return sq_accumulate_impl(p, packed_dev, charge_packed_dev, n, box, method, out_dev, stream);
}

// Direct sums over caller-defined atom groups (any order of groups, counts that change per frame):
// rho_g(k) = sum_{j in g} exp(i k.r_j) for the plan's vectors, groups contiguous in packed_dev.
extern "C" int trj_sq_rho_groups(trj_sq_plan* p, const float* packed_dev, int64_t n, const float box[3], int ngroups,
                                 const int64_t* group_off_host, double* rho_out, void* stream) {
    if (!p) return TRJ_ERR_INVALID;
    trj_ctx* ctx = p->ctx;
    if (!box || !group_off_host || !rho_out || ngroups < 1 || ngroups > 4096)
        return trj_fail(ctx, TRJ_ERR_INVALID, "sq rho groups: bad arguments (ngroups=%d)", ngroups);
    if (group_off_host[0] != 0 || group_off_host[ngroups] != n)
        return trj_fail(ctx, TRJ_ERR_INVALID, "sq rho groups: offsets must run from 0 to n=%lld", (long long)n);
    for (int g = 0; g < ngroups; ++g)
        if (group_off_host[g + 1] < group_off_host[g])
            return trj_fail(ctx, TRJ_ERR_INVALID, "sq rho groups: offsets decrease at group %d", g);
    if (n > 0 && (!packed_dev || ((uintptr_t)packed_dev) % 16))
        return trj_fail(ctx, TRJ_ERR_INVALID, "sq rho groups: packed_dev null or not 16-byte aligned");
    if (!(box[0] > 0.f && box[1] > 0.f && box[2] > 0.f))
        return trj_fail(ctx, TRJ_ERR_INVALID, "sq rho groups: box edges must be positive");
    if (p->nvec == 0) return TRJ_OK;
    trj_device_guard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    const int nsplit = plain_nsplit(ctx, p->nvec, std::max<int64_t>(n, 1));
    const size_t phase_need = sizeof(uint4) * (size_t)std::max<int64_t>(n, 1);
    const size_t part_need = sizeof(double2) * (size_t)nsplit * ngroups * p->nvec;
    const size_t rho_need = sizeof(double2) * (size_t)ngroups * p->nvec;
    const size_t off_need = sizeof(int64_t) * (size_t)(ngroups + 1);
    const size_t need = phase_need + part_need + rho_need + off_need + 4 * 256;
    if (need > p->groups_bytes) {
        if (p->groups_buf) {
            TRJ_CUDA_TRY(ctx, cudaStreamSynchronize(s));
            trj_dev_free(ctx, p->groups_buf);
            p->groups_buf = nullptr;
            p->groups_bytes = 0;
        }
        if (trj_dev_alloc(ctx, &p->groups_buf, need) != cudaSuccess)
            return trj_fail(ctx, TRJ_ERR_NOMEM, "sq rho groups: %zu bytes of scratch", need);
        p->groups_bytes = need;
    }
    auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
    char* base = (char*)p->groups_buf;
    uint4* phase = (uint4*)base;
    double2* part = (double2*)(base + align(phase_need));
    double2* rho = (double2*)(base + align(phase_need) + align(part_need));
    int64_t* off = (int64_t*)(base + align(phase_need) + align(part_need) + align(rho_need));
    // pageable source: staged before the call returns
    TRJ_CUDA_TRY(ctx, cudaMemcpyAsync(off, group_off_host, off_need, cudaMemcpyHostToDevice, s));
    if (n > 0)
        phase_coords_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>((const float4*)packed_dev, n, (double)box[0],
                                                                       (double)box[1], (double)box[2], phase, nullptr,
                                                                       p->z_from_y);
    const int vpt = plain_vpt(p->nvec);
    dim3 grid((unsigned)((p->nvec + kPlainThreads * vpt - 1) / (kPlainThreads * vpt)), (unsigned)nsplit);
    if (vpt == 1)
        sq_plain_kernel<1><<<grid, kPlainThreads, 0, s>>>(phase, off, ngroups, -1, p->vec_dev, p->plain_all_dev,
                                                          (int)p->nvec, p->nvec, nsplit, part);
    else
        sq_plain_kernel<kPlainVPT><<<grid, kPlainThreads, 0, s>>>(phase, off, ngroups, -1, p->vec_dev,
                                                                  p->plain_all_dev, (int)p->nvec, p->nvec, nsplit, part);
    const int64_t tot = p->nvec * ngroups;
    gather_plain_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(part, p->plain_all_dev, (int)p->nvec, p->nvec,
                                                                      ngroups, nsplit, rho);
    unpermute_rho_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(rho, p->vec_dev, p->nvec, ngroups,
                                                                       (double2*)rho_out);
    ctx->launches += 4;
    TRJ_CUDA_TRY(ctx, cudaGetLastError());
    return TRJ_OK;
}

extern "C" int trj_sq_kernel_ms(trj_sq_plan* p, float* ms) {
    if (!p) return TRJ_ERR_INVALID;
    return p->timer.elapsed(p->ctx, ms);
}

extern "C" int trj_sq_rho(trj_sq_plan* p, double* rho_out, void* stream) {
    if (!p) return TRJ_ERR_INVALID;
    if (!rho_out) return trj_fail(p->ctx, TRJ_ERR_INVALID, "sq rho: null output");
    if (p->last_method < 0) return trj_fail(p->ctx, TRJ_ERR_INVALID, "sq rho: no accumulate call yet");
    if (p->nvec == 0) return TRJ_OK;
    trj_device_guard g(p->ctx->device);
    int64_t tot = p->nvec * p->nsp;
    unpermute_rho_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        p->rho_dev, p->vec_dev, p->nvec, p->nsp, (double2*)rho_out);
    TRJ_CUDA_TRY(p->ctx, cudaGetLastError());
    return TRJ_OK;
}

extern "C" int trj_sq_plan_set_z_from_y(trj_sq_plan* p, int mul) {
    if (!p) return TRJ_ERR_INVALID;
    if (mul < 0 || mul > 1024) return trj_fail(p->ctx, TRJ_ERR_INVALID, "sq plan: z-from-y multiplier %d", mul);
    p->z_from_y = (unsigned)mul;
    return TRJ_OK;
}

// ---- fused multi-request launch: host side of the direct sum -----------------------------------

void trj_batch_launch_sq(BatchHeader* hdr, const BatchItem* items, const uint4* phase, int grid_sq, int grid_red,
                         cudaStream_t s) {
    batch_sq_kernel<<<grid_sq, kPlainThreads, 0, s>>>(hdr, items, phase);
    batch_reduce_kernel<<<grid_red, 256, 0, s>>>(hdr, items);
}

int trj_batch_sq_occupancy(int* per_sm_sq, int* per_sm_red) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm_sq, batch_sq_kernel, kPlainThreads, 0) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm_red, batch_reduce_kernel, 256, 0) != cudaSuccess)
        return -1;
    return 0;
}

int trj_batch_fill_sq(trj_sq_plan* p, int64_t n, BatchItem* it) {
    trj_ctx* ctx = p->ctx;
    if (p->qsp >= 0 || p->z_from_y)
        return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "batch: charged and planar-tile S(Q) plans run unfused");
    if (p->nsp > kBatchMaxSpecies)
        return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "batch: %d species (1..%d)", p->nsp, kBatchMaxSpecies);
    if (n != p->n_atoms)
        return trj_fail(ctx, TRJ_ERR_INVALID, "batch: n=%lld but the S(Q) plan's species counts sum to %lld",
                        (long long)n, (long long)p->n_atoms);
    for (int a = 0; a <= p->nsp; ++a) it->sp_off[a] = p->species_off[a];
    it->vecs = p->vec_dev;
    it->subset = p->plain_all_dev;
    it->w = p->weight_dev;
    it->bin_start = p->bin_start_dev;
    it->sp_off_dev = p->species_off_dev;
    it->part = p->part_dev;
    it->rho = p->rho_dev;
    it->nvec = (int32_t)p->nvec;
    it->nsplit = p->nsplit_all;
    it->vpt = plain_vpt(p->nvec);
    it->nbins = p->nbins;
    it->nvblk = (int32_t)((p->nvec + (int64_t)kPlainThreads * it->vpt - 1) / ((int64_t)kPlainThreads * it->vpt));
    p->last_method = TRJ_SQ_PLAIN_FP32;
    return TRJ_OK;
}
