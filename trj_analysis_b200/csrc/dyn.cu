// dyn.cu -- time correlations over multiple time origins: coherent and self intermediate
// scattering functions F(Q,t), Fs(Q,t) and the mean-squared displacement.
//
// Restates the device work of rtcorr (reference src/modules/dynamics.cuf:157-276) with the kernels
// FqtnD (:421-507) and rtcal (:510-547).  Each of nbuffer time origins ("buffers") keeps the state of
// its origin frame; every frame adds, for every buffer whose origin has been reached, one lag row:
//   F_b(k, lag)  += Re(rho_b(k, t0) conj(rho_b(k, t))),  rho_b(k, t) = sum_a bsc_a sum_{j in a} e^{i k.r_j(t)}
//   Fs_b(k, lag) += sum_j cos(k.(r_j(t) - r_j(t0)))
//   C_r,b(lag)   += sum_j |rt_j(t) - r_j(t0)|^2 / N     (rt: coordinates unwrapped per buffer)
// summed per output bin (the qw shell of k).  Which buffer takes which lag, and when a finished buffer
// is added to the totals, is the caller's bookkeeping (the origin shifting of rtcorr).
//
// Differences from the reference, by design:
// * rho_b(k, t0) is kept per buffer when the origin frame is seen, instead of being recomputed from
//   the origin positions in every later frame (FqtnD evaluates both sums for every buffer);
// * phases are exact: coordinates become 32-bit fixed-point fractions of the box (FP64, once per
//   atom and frame) and n.u wraps in integer arithmetic, so the FP32 cosine/sine always sees an
//   angle in [-pi, pi) (FqtnD feeds __cosf/__sinf FP32 phases of size |k| L);
// * sums are FP64 in a fixed order (FqtnD adds FP32 atomics);
// * lags beyond the plan's ndyn rows are not accumulated (FqtnD has no such bound and writes the row
//   after the last, i.e. the next buffer's first lag).
// The MSD arithmetic is the reference's FP32 per atom (unwrap, difference, dot product), summed in FP64.
#include <math.h>

#include <algorithm>
#include <vector>

#include "trj_common.cuh"

namespace {

constexpr int kDynThreads = 256;
constexpr int kDynVPT = 4;        // vectors per thread
constexpr int kDynChunk = 1024;   // atoms staged per pass
constexpr int kDynSub = 64;       // FP32 run length before the FP64 add
constexpr float kTwoPiOver2_32 = 1.4629180792671596e-09f;

struct DynJob {
    int buf;     // buffer index
    int lag;     // 0-based lag row of this frame
    int origin;  // this frame is the buffer's origin
    int pad;
};

__global__ void dyn_phase_kernel(const float4* __restrict__ packed, int64_t n, double Lx, double Ly, double Lz,
                                 uint4* __restrict__ u) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = packed[i];
    const double s[3] = {(double)v.x / Lx, (double)v.y / Ly, (double)v.z / Lz};
    unsigned w[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double f = s[d] - floor(s[d]);
        w[d] = (unsigned)(long long)rint(f * 4294967296.0);  // 2^32 wraps to 0
    }
    u[i] = make_uint4(w[0], w[1], w[2], (unsigned)__float_as_int(v.w));
}

// Partial rho(k) = sum_j bsc[species_j] e^{i k.r_j} over the atom range of blockIdx.y.
__global__ void __launch_bounds__(kDynThreads) dyn_rho_kernel(const uint4* __restrict__ u, int64_t n,
                                                              const float* __restrict__ bsc, int nsp,
                                                              const int4* __restrict__ vecs, int64_t nvec,
                                                              int nsplit, double2* __restrict__ part) {
    __shared__ uint4 atoms[kDynChunk];
    __shared__ float wts[kDynChunk];
    const int tid = threadIdx.x;
    unsigned nx[kDynVPT], ny[kDynVPT], nz[kDynVPT];
    int64_t vi[kDynVPT];
#pragma unroll
    for (int q = 0; q < kDynVPT; ++q) {
        vi[q] = (int64_t)blockIdx.x * kDynThreads * kDynVPT + q * kDynThreads + tid;
        const int4 v = vi[q] < nvec ? vecs[vi[q]] : make_int4(0, 0, 0, 0);
        nx[q] = (unsigned)v.x;
        ny[q] = (unsigned)v.y;
        nz[q] = (unsigned)v.z;
    }
    const int64_t a0 = n * blockIdx.y / nsplit, a1 = n * (blockIdx.y + 1) / nsplit;
    double accr[kDynVPT], acci[kDynVPT];
#pragma unroll
    for (int q = 0; q < kDynVPT; ++q) accr[q] = acci[q] = 0.0;
    for (int64_t c0 = a0; c0 < a1; c0 += kDynChunk) {
        const int cnt = (int)min((int64_t)kDynChunk, a1 - c0);
        __syncthreads();
        for (int k = tid; k < cnt; k += kDynThreads) {
            const uint4 a = u[c0 + k];
            atoms[k] = a;
            const int s = (int)a.w;
            wts[k] = (s >= 0 && s < nsp) ? bsc[s] : 0.f;
        }
        __syncthreads();
        for (int j0 = 0; j0 < cnt; j0 += kDynSub) {
            const int j1 = min(cnt, j0 + kDynSub);
            float fr[kDynVPT], fi[kDynVPT];
#pragma unroll
            for (int q = 0; q < kDynVPT; ++q) fr[q] = fi[q] = 0.f;
            for (int j = j0; j < j1; ++j) {
                const uint4 a = atoms[j];
                const float w = wts[j];
#pragma unroll
                for (int q = 0; q < kDynVPT; ++q) {
                    const unsigned ph = nx[q] * a.x + ny[q] * a.y + nz[q] * a.z;
                    float sn, cs;
                    __sincosf(__int2float_rn((int)ph) * kTwoPiOver2_32, &sn, &cs);
                    fr[q] = fmaf(w, cs, fr[q]);
                    fi[q] = fmaf(w, sn, fi[q]);
                }
            }
#pragma unroll
            for (int q = 0; q < kDynVPT; ++q) {
                accr[q] += (double)fr[q];
                acci[q] += (double)fi[q];
            }
        }
    }
#pragma unroll
    for (int q = 0; q < kDynVPT; ++q)
        if (vi[q] < nvec) part[(int64_t)blockIdx.y * nvec + vi[q]] = make_double2(accr[q], acci[q]);
}

// rho_t = sum over splits (fixed order); origin buffers keep a copy as their rho(k, t0).
__global__ void dyn_rho_gather_kernel(const double2* __restrict__ part, int64_t nvec, int nsplit,
                                      const DynJob* __restrict__ jobs, int njobs, double2* __restrict__ rho_t,
                                      double2* __restrict__ rho0) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nvec) return;
    double re = 0.0, im = 0.0;
    for (int s = 0; s < nsplit; ++s) {
        const double2 p = part[(int64_t)s * nvec + k];
        re += p.x;
        im += p.y;
    }
    rho_t[k] = make_double2(re, im);
    for (int j = 0; j < njobs; ++j)
        if (jobs[j].origin) rho0[(int64_t)jobs[j].buf * nvec + k] = make_double2(re, im);
}

// Origin frames: phases and coordinates of every atom become the buffer's origin state.
__global__ void dyn_origin_kernel(const float4* __restrict__ packed, const uint4* __restrict__ u, int64_t n,
                                  const DynJob* __restrict__ jobs, uint4* __restrict__ u0,
                                  float4* __restrict__ r0, float4* __restrict__ rt) {
    const DynJob jb = jobs[blockIdx.y];
    if (!jb.origin) return;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t o = (int64_t)jb.buf * n + i;
    const float4 v = packed[i];
    u0[o] = u[i];
    r0[o] = v;
    rt[o] = v;
}

// rtcal (dynamics.cuf:510-547): unwrap rt toward the current frame, FP32 |rt - r0|^2 per atom,
// FP64 block sums (written per block, reduced in a fixed order later).
__global__ void dyn_msd_kernel(const float4* __restrict__ packed, int64_t n, float Lx, float Ly, float Lz,
                               const DynJob* __restrict__ jobs, const float4* __restrict__ r0,
                               float4* __restrict__ rt, double* __restrict__ msd_part) {
    __shared__ double red[kDynThreads / 32];
    const DynJob jb = jobs[blockIdx.y];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double s = 0.0;
    if (i < n) {
        const int64_t o = (int64_t)jb.buf * n + i;
        const float4 r = packed[i];
        float4 t = rt[o];
        const float L[3] = {Lx, Ly, Lz};
        float rc[3] = {r.x, r.y, r.z}, tc[3] = {t.x, t.y, t.z};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            // rt = r + L*nint((rt - r)/L), each FP32 operation rounded once (nint: half away from zero)
            const float m = roundf(__fdiv_rn(__fsub_rn(tc[d], rc[d]), L[d]));
            tc[d] = __fadd_rn(rc[d], __fmul_rn(L[d], m));
        }
        t.x = tc[0];
        t.y = tc[1];
        t.z = tc[2];
        rt[o] = t;
        const float4 z = r0[o];
        const float dx = __fsub_rn(t.x, z.x), dy = __fsub_rn(t.y, z.y), dz = __fsub_rn(t.z, z.z);
        s = (double)__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    }
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        msd_part[(int64_t)blockIdx.y * gridDim.x + blockIdx.x] = t;
    }
}

// Partial Fs(k) = sum_j cos(k.(r_j(t) - r_j(t0))) over the atom range of blockIdx.y, for job blockIdx.z.
__global__ void __launch_bounds__(kDynThreads) dyn_self_kernel(const uint4* __restrict__ u,
                                                               const uint4* __restrict__ u0, int64_t n,
                                                               const DynJob* __restrict__ jobs,
                                                               const int4* __restrict__ vecs, int64_t nvec,
                                                               int nsplit, double* __restrict__ part) {
    __shared__ uint4 dis[kDynChunk];
    const int tid = threadIdx.x;
    const DynJob jb = jobs[blockIdx.z];
    const uint4* __restrict__ org = u0 + (int64_t)jb.buf * n;
    unsigned nx[kDynVPT], ny[kDynVPT], nz[kDynVPT];
    int64_t vi[kDynVPT];
#pragma unroll
    for (int q = 0; q < kDynVPT; ++q) {
        vi[q] = (int64_t)blockIdx.x * kDynThreads * kDynVPT + q * kDynThreads + tid;
        const int4 v = vi[q] < nvec ? vecs[vi[q]] : make_int4(0, 0, 0, 0);
        nx[q] = (unsigned)v.x;
        ny[q] = (unsigned)v.y;
        nz[q] = (unsigned)v.z;
    }
    const int64_t a0 = n * blockIdx.y / nsplit, a1 = n * (blockIdx.y + 1) / nsplit;
    double acc[kDynVPT];
#pragma unroll
    for (int q = 0; q < kDynVPT; ++q) acc[q] = 0.0;
    for (int64_t c0 = a0; c0 < a1; c0 += kDynChunk) {
        const int cnt = (int)min((int64_t)kDynChunk, a1 - c0);
        __syncthreads();
        for (int k = tid; k < cnt; k += kDynThreads) {
            const uint4 a = u[c0 + k], b = org[c0 + k];
            dis[k] = make_uint4(a.x - b.x, a.y - b.y, a.z - b.z, 0u);  // displacement, exact mod 1 box
        }
        __syncthreads();
        for (int j0 = 0; j0 < cnt; j0 += kDynSub) {
            const int j1 = min(cnt, j0 + kDynSub);
            float f[kDynVPT];
#pragma unroll
            for (int q = 0; q < kDynVPT; ++q) f[q] = 0.f;
            for (int j = j0; j < j1; ++j) {
                const uint4 d = dis[j];
#pragma unroll
                for (int q = 0; q < kDynVPT; ++q) {
                    const unsigned ph = nx[q] * d.x + ny[q] * d.y + nz[q] * d.z;
                    f[q] += __cosf(__int2float_rn((int)ph) * kTwoPiOver2_32);
                }
            }
#pragma unroll
            for (int q = 0; q < kDynVPT; ++q) acc[q] += (double)f[q];
        }
    }
#pragma unroll
    for (int q = 0; q < kDynVPT; ++q)
        if (vi[q] < nvec) part[((int64_t)blockIdx.z * nsplit + blockIdx.y) * nvec + vi[q]] = acc[q];
}

// One block per (bin, job): the bin's vectors in a fixed order; bin 0's block also adds the MSD.
__global__ void dyn_reduce_kernel(const double* __restrict__ self_part, const double2* __restrict__ rho_t,
                                  const double2* __restrict__ rho0, const int32_t* __restrict__ bin_start,
                                  const int32_t* __restrict__ bin_vec, int64_t nvec, int nsplit, int nbins,
                                  int ndyn, const DynJob* __restrict__ jobs, const double* __restrict__ msd_part,
                                  int msd_blocks, int64_t n, double* __restrict__ fc, double* __restrict__ fs,
                                  double* __restrict__ msd) {
    __shared__ double red[2][kDynThreads / 32];
    const int bin = blockIdx.x, j = blockIdx.y;
    const DynJob jb = jobs[j];
    const int v0 = bin_start[bin], v1 = bin_start[bin + 1];
    double sc = 0.0, ss = 0.0;
    for (int t = v0 + threadIdx.x; t < v1; t += blockDim.x) {
        const int k = bin_vec[t];
        const double2 a = rho0[(int64_t)jb.buf * nvec + k], b = rho_t[k];
        sc += a.x * b.x + a.y * b.y;
        double s = 0.0;
        for (int p = 0; p < nsplit; ++p) s += self_part[((int64_t)j * nsplit + p) * nvec + k];
        ss += s;
    }
    for (int off = 16; off > 0; off >>= 1) {
        sc += __shfl_down_sync(0xffffffffu, sc, off);
        ss += __shfl_down_sync(0xffffffffu, ss, off);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = sc;
        red[1][threadIdx.x >> 5] = ss;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tc = 0.0, ts = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            tc += red[0][w];
            ts += red[1][w];
        }
        const int64_t o = ((int64_t)jb.buf * ndyn + jb.lag) * nbins + bin;
        fc[o] += tc;
        fs[o] += ts;
        if (bin == 0) {
            double m = 0.0;
            for (int b = 0; b < msd_blocks; ++b) m += msd_part[(int64_t)j * msd_blocks + b];
            msd[(int64_t)jb.buf * ndyn + jb.lag] += m / (double)n;
        }
    }
}

// Finished buffers: their rows are added to the totals and cleared (rtcorr, dynamics.cuf:250-268).
__global__ void dyn_flush_kernel(const int32_t* __restrict__ done, int ndone, int ndyn, int nbins,
                                 double* __restrict__ fc, double* __restrict__ fs, double* __restrict__ msd,
                                 double* __restrict__ fkt, double* __restrict__ fskt, double* __restrict__ r2t) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t rows = (int64_t)ndyn * nbins;
    if (e < rows) {
        double c = fkt[e], s = fskt[e];
        for (int d = 0; d < ndone; ++d) {
            const int64_t o = (int64_t)done[d] * rows + e;
            c += fc[o];
            s += fs[o];
            fc[o] = 0.0;
            fs[o] = 0.0;
        }
        fkt[e] = c;
        fskt[e] = s;
    }
    if (e < ndyn) {
        double m = r2t[e];
        for (int d = 0; d < ndone; ++d) {
            const int64_t o = (int64_t)done[d] * ndyn + e;
            m += msd[o];
            msd[o] = 0.0;
        }
        r2t[e] = m;
    }
}

}  // namespace

struct trj_dyn_plan {
    trj_ctx* ctx = nullptr;
    int nsp = 0, nbuf = 0, ndyn = 0, nbins = 0;
    int64_t n = 0, nvec = 0;
    int gx = 1;              // vector blocks of the rho/self kernels
    int nsplit_rho = 1;
    int nsplit_cap = 1;      // self-part rows: nsplit * jobs <= nsplit_cap
    int4* vecs = nullptr;
    int32_t* bin_start = nullptr;  // nbins + 1
    int32_t* bin_vec = nullptr;    // vectors of each bin
    float* bsc = nullptr;
    uint4* u = nullptr;            // n
    uint4* u0 = nullptr;           // nbuf * n
    float4* r0 = nullptr;          // nbuf * n
    float4* rt = nullptr;          // nbuf * n
    double2* rho_part = nullptr;   // nsplit_rho * nvec
    double2* rho_t = nullptr;      // nvec
    double2* rho0 = nullptr;       // nbuf * nvec
    double* self_part = nullptr;   // nsplit_cap * nvec
    double* msd_part = nullptr;    // nbuf * msd_blocks
    double* fc = nullptr;          // nbuf * ndyn * nbins
    double* fs = nullptr;          // nbuf * ndyn * nbins
    double* msd = nullptr;         // nbuf * ndyn
    DynJob* jobs_dev = nullptr;    // nbuf
    int32_t* done_dev = nullptr;   // nbuf
    std::vector<void*> blocks;
    int64_t scratch_bytes = 0;
    trj_kernel_timer timer;        // around the self kernel
};

static void dyn_free(trj_dyn_plan* p) {
    trj_device_guard g(p->ctx->device);
    for (void* b : p->blocks) trj_dev_free(p->ctx, b);
    p->blocks.clear();
    p->timer.release();
}

template <class T>
static bool dyn_alloc(trj_dyn_plan* p, T** out, size_t count) {
    const size_t bytes = std::max<size_t>(1, count) * sizeof(T);
    void* q = nullptr;
    if (trj_dev_alloc(p->ctx, &q, bytes) != cudaSuccess) return false;
    p->blocks.push_back(q);
    p->scratch_bytes += (int64_t)bytes;
    *out = reinterpret_cast<T*>(q);
    return true;
}

extern "C" int trj_dyn_plan_create(trj_ctx* ctx, int nsp, int64_t n, int nbuffer, int ndyn, int64_t nvec,
                                   const int32_t* vec_host, const int32_t* bin_host, int nbins,
                                   const float* bsc_host, trj_dyn_plan** out) {
    if (!ctx || !out) return TRJ_ERR_INVALID;
    *out = nullptr;
    if (nsp < 1 || nsp > 16) return trj_fail(ctx, TRJ_ERR_INVALID, "dyn plan: nsp=%d (1..16)", nsp);
    if (n < 1 || n > (int64_t)INT32_MAX) return trj_fail(ctx, TRJ_ERR_INVALID, "dyn plan: n=%lld", (long long)n);
    if (nbuffer < 1 || nbuffer > 65535 || ndyn < 1 || nbins < 1)
        return trj_fail(ctx, TRJ_ERR_INVALID, "dyn plan: nbuffer=%d ndyn=%d nbins=%d", nbuffer, ndyn, nbins);
    if (nvec < 0 || nvec > (int64_t)INT32_MAX / 2 || (nvec > 0 && (!vec_host || !bin_host)) || !bsc_host)
        return trj_fail(ctx, TRJ_ERR_INVALID, "dyn plan: vectors");
    for (int64_t v = 0; v < nvec; ++v)
        if (bin_host[v] < 0 || bin_host[v] >= nbins)
            return trj_fail(ctx, TRJ_ERR_INVALID, "dyn plan: vector %lld has bin %d outside 0..%d", (long long)v,
                            bin_host[v], nbins - 1);
    trj_dyn_plan* p = new trj_dyn_plan();
    p->ctx = ctx;
    p->nsp = nsp;
    p->n = n;
    p->nbuf = nbuffer;
    p->ndyn = ndyn;
    p->nbins = nbins;
    p->nvec = nvec;
    p->gx = (int)std::max<int64_t>(1, (nvec + kDynThreads * kDynVPT - 1) / (kDynThreads * kDynVPT));
    const int64_t target = (int64_t)ctx->sm_count * 8;
    const int64_t by_atoms = std::max<int64_t>(1, n / kDynChunk);
    p->nsplit_rho = (int)std::min<int64_t>(by_atoms, std::max<int64_t>(1, (target + p->gx - 1) / p->gx));
    // self-term partial rows (splits x buffers): enough for every buffer to split as far as the atoms
    // allow, within 256 MB of partials
    const int64_t split_max = std::min<int64_t>(by_atoms, target);
    const int64_t rows_budget = std::max<int64_t>(nbuffer, ((int64_t)256 << 20) / (8 * std::max<int64_t>(nvec, 1)));
    p->nsplit_cap = (int)std::min<int64_t>((int64_t)nbuffer * split_max, std::max<int64_t>(rows_budget, nbuffer));
    std::vector<int4> vecs(nvec);
    std::vector<int32_t> start(nbins + 1, 0), bv(nvec);
    for (int64_t v = 0; v < nvec; ++v) {
        vecs[v] = make_int4(vec_host[3 * v], vec_host[3 * v + 1], vec_host[3 * v + 2], bin_host[v]);
        start[bin_host[v] + 1] += 1;
    }
    for (int b = 0; b < nbins; ++b) start[b + 1] += start[b];
    {
        std::vector<int32_t> fill(start.begin(), start.end() - 1);
        for (int64_t v = 0; v < nvec; ++v) bv[fill[bin_host[v]]++] = (int32_t)v;
    }
    trj_device_guard g(ctx->device);
    const int msd_blocks = (int)((n + kDynThreads - 1) / kDynThreads);
    const int64_t rows = (int64_t)nbuffer * ndyn;
    bool ok = dyn_alloc(p, &p->vecs, nvec) && dyn_alloc(p, &p->bin_start, nbins + 1) &&
              dyn_alloc(p, &p->bin_vec, nvec) && dyn_alloc(p, &p->bsc, nsp) && dyn_alloc(p, &p->u, n) &&
              dyn_alloc(p, &p->u0, (size_t)nbuffer * n) && dyn_alloc(p, &p->r0, (size_t)nbuffer * n) &&
              dyn_alloc(p, &p->rt, (size_t)nbuffer * n) &&
              dyn_alloc(p, &p->rho_part, (size_t)p->nsplit_rho * nvec) && dyn_alloc(p, &p->rho_t, nvec) &&
              dyn_alloc(p, &p->rho0, (size_t)nbuffer * nvec) &&
              dyn_alloc(p, &p->self_part, (size_t)p->nsplit_cap * nvec) &&
              dyn_alloc(p, &p->msd_part, (size_t)nbuffer * msd_blocks) &&
              dyn_alloc(p, &p->fc, (size_t)rows * nbins) && dyn_alloc(p, &p->fs, (size_t)rows * nbins) &&
              dyn_alloc(p, &p->msd, rows) && dyn_alloc(p, &p->jobs_dev, nbuffer) &&
              dyn_alloc(p, &p->done_dev, nbuffer);
    if (!ok) {
        dyn_free(p);
        delete p;
        return trj_fail(ctx, TRJ_ERR_NOMEM, "dyn plan: device allocation failed (nbuffer=%d, n=%lld)", nbuffer,
                        (long long)n);
    }
    cudaError_t e = cudaSuccess;
    if (nvec) {
        e = cudaMemcpy(p->vecs, vecs.data(), sizeof(int4) * nvec, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(p->bin_vec, bv.data(), sizeof(int32_t) * nvec, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(p->bin_start, start.data(), sizeof(int32_t) * (nbins + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->bsc, bsc_host, sizeof(float) * nsp, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(p->fc, 0, sizeof(double) * rows * nbins);
    if (e == cudaSuccess) e = cudaMemset(p->fs, 0, sizeof(double) * rows * nbins);
    if (e == cudaSuccess) e = cudaMemset(p->msd, 0, sizeof(double) * rows);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        dyn_free(p);
        delete p;
        return trj_fail(ctx, TRJ_ERR_CUDA, "dyn plan: %s", cudaGetErrorString(e));
    }
    *out = p;
    return TRJ_OK;
}

extern "C" int trj_dyn_plan_info(const trj_dyn_plan* p, int64_t* scratch_bytes) {
    if (!p) return TRJ_ERR_INVALID;
    if (scratch_bytes) *scratch_bytes = p->scratch_bytes;
    return TRJ_OK;
}

extern "C" int trj_dyn_accumulate(trj_dyn_plan* p, const float* packed_dev, int64_t n, const float box[3],
                                  const int32_t* lag_host, const uint8_t* origin_host, void* stream) {
    if (!p) return TRJ_ERR_INVALID;
    trj_ctx* ctx = p->ctx;
    if (!box || !lag_host || !origin_host) return trj_fail(ctx, TRJ_ERR_INVALID, "dyn accumulate: null argument");
    if (n != p->n)
        return trj_fail(ctx, TRJ_ERR_INVALID, "dyn accumulate: n=%lld, plan made for %lld atoms", (long long)n,
                        (long long)p->n);
    if (!packed_dev || ((uintptr_t)packed_dev) % 16)
        return trj_fail(ctx, TRJ_ERR_INVALID, "dyn accumulate: packed_dev null or not 16-byte aligned");
    if (!(box[0] > 0.f && box[1] > 0.f && box[2] > 0.f))
        return trj_fail(ctx, TRJ_ERR_INVALID, "dyn accumulate: box edges must be positive");
    std::vector<DynJob> jobs;
    for (int b = 0; b < p->nbuf; ++b) {
        const int lag = lag_host[b];
        if (lag < 0) continue;
        if (lag >= p->ndyn)
            return trj_fail(ctx, TRJ_ERR_INVALID, "dyn accumulate: buffer %d lag %d outside 0..%d", b, lag,
                            p->ndyn - 1);
        if (origin_host[b] && lag != 0)
            return trj_fail(ctx, TRJ_ERR_INVALID, "dyn accumulate: buffer %d starts at lag %d (must be 0)", b, lag);
        jobs.push_back(DynJob{b, lag, origin_host[b] ? 1 : 0, 0});
    }
    if (jobs.empty()) return TRJ_OK;
    trj_device_guard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    const int nj = (int)jobs.size();
    // pageable source: the call returns after the bytes are staged, so the vector may go out of scope
    TRJ_CUDA_TRY(ctx, cudaMemcpyAsync(p->jobs_dev, jobs.data(), sizeof(DynJob) * nj, cudaMemcpyHostToDevice, s));
    const unsigned nb = (unsigned)((n + kDynThreads - 1) / kDynThreads);
    dyn_phase_kernel<<<nb, kDynThreads, 0, s>>>((const float4*)packed_dev, n, (double)box[0], (double)box[1],
                                                 (double)box[2], p->u);
    int launches = 1;
    if (p->nvec > 0) {
        dyn_rho_kernel<<<dim3(p->gx, p->nsplit_rho), kDynThreads, 0, s>>>(p->u, n, p->bsc, p->nsp, p->vecs, p->nvec,
                                                                          p->nsplit_rho, p->rho_part);
        dyn_rho_gather_kernel<<<(unsigned)((p->nvec + 255) / 256), 256, 0, s>>>(p->rho_part, p->nvec, p->nsplit_rho,
                                                                               p->jobs_dev, nj, p->rho_t, p->rho0);
        launches += 2;
    }
    dyn_origin_kernel<<<dim3(nb, nj), kDynThreads, 0, s>>>((const float4*)packed_dev, p->u, n, p->jobs_dev, p->u0,
                                                          p->r0, p->rt);
    dyn_msd_kernel<<<dim3(nb, nj), kDynThreads, 0, s>>>((const float4*)packed_dev, n, box[0], box[1], box[2],
                                                       p->jobs_dev, p->r0, p->rt, p->msd_part);
    launches += 2;
    const int64_t target = (int64_t)ctx->sm_count * 8;
    const int64_t by_atoms = std::max<int64_t>(1, n / kDynChunk);
    int nsplit = (int)std::min<int64_t>(by_atoms, std::max<int64_t>(1, (target + (int64_t)p->gx * nj - 1) /
                                                                          ((int64_t)p->gx * nj)));
    nsplit = std::max(1, std::min(nsplit, p->nsplit_cap / nj));
    if (p->nvec > 0) {
        p->timer.begin(ctx, s);
        dyn_self_kernel<<<dim3(p->gx, nsplit, nj), kDynThreads, 0, s>>>(p->u, p->u0, n, p->jobs_dev, p->vecs,
                                                                        p->nvec, nsplit, p->self_part);
        p->timer.end(ctx, s);
        launches += 1;
    }
    dyn_reduce_kernel<<<dim3(p->nbins, nj), kDynThreads, 0, s>>>(p->self_part, p->rho_t, p->rho0, p->bin_start,
                                                                 p->bin_vec, p->nvec, nsplit, p->nbins, p->ndyn,
                                                                 p->jobs_dev, p->msd_part, (int)nb, n, p->fc, p->fs,
                                                                 p->msd);
    launches += 1;
    ctx->launches += launches;
    TRJ_CUDA_TRY(ctx, cudaGetLastError());
    return TRJ_OK;
}

extern "C" int trj_dyn_flush(trj_dyn_plan* p, const uint8_t* done_host, double* fkt_dev, double* fskt_dev,
                             double* r2t_dev, void* stream) {
    if (!p) return TRJ_ERR_INVALID;
    trj_ctx* ctx = p->ctx;
    if (!done_host || !fkt_dev || !fskt_dev || !r2t_dev)
        return trj_fail(ctx, TRJ_ERR_INVALID, "dyn flush: null argument");
    std::vector<int32_t> done;
    for (int b = 0; b < p->nbuf; ++b)
        if (done_host[b]) done.push_back(b);
    if (done.empty()) return TRJ_OK;
    trj_device_guard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    TRJ_CUDA_TRY(ctx, cudaMemcpyAsync(p->done_dev, done.data(), sizeof(int32_t) * done.size(), cudaMemcpyHostToDevice,
                                      s));
    const int64_t rows = std::max<int64_t>((int64_t)p->ndyn * p->nbins, p->ndyn);
    dyn_flush_kernel<<<(unsigned)((rows + 255) / 256), 256, 0, s>>>(p->done_dev, (int)done.size(), p->ndyn, p->nbins,
                                                                   p->fc, p->fs, p->msd, fkt_dev, fskt_dev, r2t_dev);
    ctx->launches += 1;
    TRJ_CUDA_TRY(ctx, cudaGetLastError());
    return TRJ_OK;
}

extern "C" int trj_dyn_kernel_ms(trj_dyn_plan* p, float* ms) {
    if (!p) return TRJ_ERR_INVALID;
    return p->timer.elapsed(p->ctx, ms);
}

extern "C" int trj_dyn_plan_destroy(trj_dyn_plan* p) {
    if (!p) return TRJ_OK;
    dyn_free(p);
    delete p;
    return TRJ_OK;
}
