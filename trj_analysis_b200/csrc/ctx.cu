// ctx.cu -- context, error reporting, and the device frame-layout step.
//
// The layout step restates select_ncdfinput (reference src/core/netcdf.f90:582-692):
// species-contiguous order (stable within a species, netcdf.f90:625-687) and the
// periodic fold r = r - L*int(r/L) (netcdf.f90:681), both on the device.
#include <stdarg.h>

#include <mutex>

#include "batch.cuh"
#include "trj_common.cuh"

int trj_fail(trj_ctx* ctx, int code, const char* fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->last_error = buf;
    }
    return code;
}

extern "C" int trj_abi_version(void) { return TRJ_ABI_VERSION; }

extern "C" int trj_ctx_create(int device, trj_ctx** out) {
    if (!out) return TRJ_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return TRJ_ERR_CUDA;
    }
    if (device < 0 || device >= ndev) return TRJ_ERR_INVALID;
    trj_ctx* ctx = new trj_ctx();
    ctx->device = device;
    trj_device_guard g(device);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        delete ctx;
        return TRJ_ERR_CUDA;
    }
    if (prop.major != 10) {
        // This build carries sm_100a code only.
        delete ctx;
        return TRJ_ERR_UNSUPPORTED;
    }
    ctx->sm_count = prop.multiProcessorCount;
    ctx->smem_optin = prop.sharedMemPerBlockOptin;
    if (cudaMalloc(&ctx->status_dev, 8 * sizeof(unsigned)) != cudaSuccess ||
        cudaMallocHost(&ctx->status_host, 8 * sizeof(unsigned)) != cudaSuccess) {
        if (ctx->status_dev) cudaFree(ctx->status_dev);
        delete ctx;
        return TRJ_ERR_NOMEM;
    }
    cudaMemset(ctx->status_dev, 0, 8 * sizeof(unsigned));
    cudaDeviceSynchronize();
    *out = ctx;
    return TRJ_OK;
}

extern "C" int trj_ctx_destroy(trj_ctx* ctx) {
    if (!ctx) return TRJ_OK;
    {
        trj_device_guard g(ctx->device);
        if (ctx->status_dev) cudaFree(ctx->status_dev);
        if (ctx->status_host) cudaFreeHost(ctx->status_host);
        // a caller allocator's free callback takes no stream: layout kernels still in flight finish first
        if (ctx->alloc && !ctx->pack_scratch.empty()) cudaDeviceSynchronize();
        for (auto& kv : ctx->pack_scratch) trj_dev_free(ctx, kv.second.ptr);
        ctx->pack_scratch.clear();
    }
    delete ctx;
    return TRJ_OK;
}

extern "C" const char* trj_ctx_last_error(const trj_ctx* ctx) {
    return ctx ? ctx->last_error.c_str() : "null context";
}

extern "C" int trj_ctx_sm_count(const trj_ctx* ctx) { return ctx ? ctx->sm_count : 0; }

extern "C" int trj_ctx_set_allocator(trj_ctx* ctx, trj_alloc_fn alloc, trj_free_fn free_fn, void* user) {
    if (!ctx) return TRJ_ERR_INVALID;
    if ((alloc == nullptr) != (free_fn == nullptr))
        return trj_fail(ctx, TRJ_ERR_INVALID, "trj_ctx_set_allocator: give both callbacks or neither");
    if (!ctx->pack_scratch.empty()) {
        // Layout kernels on any stream may still use the scratch; the caller's free callback takes no
        // stream, so nothing may be handed back to it before they finish.
        trj_device_guard g(ctx->device);
        TRJ_CUDA_TRY(ctx, cudaDeviceSynchronize());
    }
    for (auto& kv : ctx->pack_scratch) trj_dev_free(ctx, kv.second.ptr);  // with the allocator that made it
    ctx->pack_scratch.clear();
    ctx->alloc = alloc;
    ctx->free_fn = free_fn;
    ctx->alloc_user = user;
    return TRJ_OK;
}

extern "C" int64_t trj_ctx_launches(const trj_ctx* ctx) { return ctx ? ctx->launches : 0; }

extern "C" int trj_ctx_set_sq_tile_cols(trj_ctx* ctx, int cols) {
    if (!ctx) return TRJ_ERR_INVALID;
    if (cols != 0 && (cols < 32 || cols > 224 || cols % 16 != 0))
        return trj_fail(ctx, TRJ_ERR_INVALID, "trj_ctx_set_sq_tile_cols: %d (0, or 32..224 in steps of 16)", cols);
    ctx->sq_tile_cols = cols;
    return TRJ_OK;
}

extern "C" int trj_ctx_set_timing(trj_ctx* ctx, int enable) {
    if (!ctx) return TRJ_ERR_INVALID;
    ctx->timing = enable != 0;
    return TRJ_OK;
}

int trj_kernel_timer::elapsed(trj_ctx* ctx, float* ms) {
    if (!ms) return trj_fail(ctx, TRJ_ERR_INVALID, "kernel_ms: null output");
    if (!recorded) return trj_fail(ctx, TRJ_ERR_INVALID, "kernel_ms: no timed launch (enable timing first)");
    trj_device_guard g(ctx->device);
    TRJ_CUDA_TRY(ctx, cudaEventSynchronize(stop));
    TRJ_CUDA_TRY(ctx, cudaEventElapsedTime(ms, start, stop));
    return TRJ_OK;
}

extern "C" int trj_ctx_check(trj_ctx* ctx, void* stream) {
    if (!ctx) return TRJ_ERR_INVALID;
    trj_device_guard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    TRJ_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->status_host, ctx->status_dev, 8 * sizeof(unsigned),
                                      cudaMemcpyDeviceToHost, s));
    TRJ_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    unsigned st = ctx->status_host[0];
    if (st) TRJ_CUDA_TRY(ctx, cudaMemsetAsync(ctx->status_dev, 0, 8 * sizeof(unsigned), s));
    if (st & TRJ_DEV_TIMEOUT)
        return trj_fail(ctx, TRJ_ERR_TIMEOUT, "device-side bounded wait timed out (status 0x%x)", st);
    if (st & TRJ_DEV_BAD_DATA)
        return trj_fail(ctx, TRJ_ERR_DATA, "non-finite coordinate or species index out of range");
    if (st & TRJ_DEV_COUNT_MISMATCH)
        return trj_fail(ctx, TRJ_ERR_DATA, "species counts of the frame differ from the plan's");
    if (st & TRJ_DEV_CAPACITY)
        return trj_fail(ctx, TRJ_ERR_CAPACITY, "device-side capacity exceeded (status 0x%x)", st);
    return TRJ_OK;
}

// ---------------------------------------------------------------------------
// Frame layout: fold + stable species partition.
// ---------------------------------------------------------------------------

namespace {

constexpr int kPackThreads = 256;
constexpr int kPackRounds = 4;
constexpr int kPackChunk = kPackThreads * kPackRounds;  // atoms per block
constexpr int kMaxSpecies = 16;

// Species of atom i: sp[i], or lut[sp[i]] when a type-to-species table is given (-1: invalid).
__device__ __forceinline__ int species_of(const int32_t* __restrict__ sp, int64_t i, const int32_t* __restrict__ lut,
                                          int nlut) {
    const int t = sp[i];
    if (!lut) return t;
    return (t >= 0 && t < nlut) ? lut[t] : -1;
}

__global__ void pack_count_kernel(const float* __restrict__ xyz, const int32_t* __restrict__ sp,
                                  int64_t n, int nsp, int32_t* __restrict__ block_counts,
                                  unsigned* status, const int32_t* __restrict__ lut, int nlut) {
    __shared__ int cnt[kMaxSpecies];
    if (threadIdx.x < kMaxSpecies) cnt[threadIdx.x] = 0;
    __syncthreads();
    int64_t base = (int64_t)blockIdx.x * kPackChunk;
    bool bad = false;
    for (int r = 0; r < kPackRounds; ++r) {
        int64_t i = base + r * kPackThreads + threadIdx.x;
        if (i < n) {
            int s = species_of(sp, i, lut, nlut);
            float x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
            if (s < 0 || s >= nsp || !isfinite(x) || !isfinite(y) || !isfinite(z)) bad = true;
            if (s >= 0 && s < nsp) atomicAdd(&cnt[s], 1);
        }
    }
    if (bad) trj_raise(status, TRJ_DEV_BAD_DATA);
    __syncthreads();
    if (threadIdx.x < nsp) block_counts[(int64_t)blockIdx.x * nsp + threadIdx.x] = cnt[threadIdx.x];
}

// One block: exclusive scan of per-block counts, species after species.
__global__ void pack_scan_kernel(int32_t* __restrict__ block_counts, int64_t nblocks, int nsp,
                                 int64_t* __restrict__ counts_out, int64_t* __restrict__ block_base) {
    __shared__ int64_t partial[1024];
    __shared__ int64_t species_base;
    if (threadIdx.x == 0) species_base = 0;
    __syncthreads();
    int64_t per = (nblocks + blockDim.x - 1) / blockDim.x;
    for (int s = 0; s < nsp; ++s) {
        int64_t b0 = threadIdx.x * per, b1 = b0 + per < nblocks ? b0 + per : nblocks;
        int64_t sum = 0;
        for (int64_t b = b0; b < b1; ++b) sum += block_counts[b * nsp + s];
        partial[threadIdx.x] = sum;
        __syncthreads();
        if (threadIdx.x == 0) {
            int64_t run = 0;
            for (unsigned t = 0; t < blockDim.x; ++t) {
                int64_t v = partial[t];
                partial[t] = run;
                run += v;
            }
            counts_out[s] = run;
        }
        __syncthreads();
        int64_t run = species_base + partial[threadIdx.x];
        for (int64_t b = b0; b < b1; ++b) {
            block_base[b * nsp + s] = run;
            run += block_counts[b * nsp + s];
        }
        __syncthreads();
        if (threadIdx.x == 0) species_base += counts_out[s];
        __syncthreads();
    }
}

__global__ void pack_scatter_kernel(const float* __restrict__ xyz, const int32_t* __restrict__ sp,
                                    int64_t n, int nsp, float Lx, float Ly, float Lz,
                                    const int64_t* __restrict__ block_base,
                                    float4* __restrict__ packed, const float* __restrict__ q,
                                    float* __restrict__ qpacked, const int32_t* __restrict__ lut, int nlut) {
    __shared__ int64_t base[kMaxSpecies];
    __shared__ int warp_cnt[kPackThreads / 32][kMaxSpecies];
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (threadIdx.x < nsp) base[threadIdx.x] = block_base[(int64_t)blockIdx.x * nsp + threadIdx.x];
    for (int k = threadIdx.x; k < (kPackThreads / 32) * kMaxSpecies; k += blockDim.x)
        (&warp_cnt[0][0])[k] = 0;
    __syncthreads();
    const unsigned lt_mask = (1u << lane) - 1u;
    int64_t start = (int64_t)blockIdx.x * kPackChunk;
    for (int r = 0; r < kPackRounds; ++r) {
        int64_t i = start + r * kPackThreads + threadIdx.x;
        int s = -1;
        if (i < n) {
            s = species_of(sp, i, lut, nlut);
            if (s < 0 || s >= nsp) s = -1;  // flagged by pack_count_kernel; dropped here
        }
        unsigned peers = __match_any_sync(0xffffffffu, s);
        int rank = __popc(peers & lt_mask);
        if (s >= 0 && rank == 0) warp_cnt[warp][s] = __popc(peers);
        __syncthreads();
        if (s >= 0) {
            int64_t off = base[s];
            for (int w = 0; w < warp; ++w) off += warp_cnt[w][s];
            off += rank;
            float4 v;
            v.x = trj_fold_ref(xyz[3 * i], Lx);
            v.y = trj_fold_ref(xyz[3 * i + 1], Ly);
            v.z = trj_fold_ref(xyz[3 * i + 2], Lz);
            v.w = __int_as_float(s);
            packed[off] = v;
            if (q) qpacked[off] = q[i];  // charges follow their atoms (netcdf.f90:656-658)
        }
        __syncthreads();
        if (threadIdx.x < nsp) {
            int tot = 0;
            for (int w = 0; w < kPackThreads / 32; ++w) {
                tot += warp_cnt[w][threadIdx.x];
                warp_cnt[w][threadIdx.x] = 0;
            }
            base[threadIdx.x] += tot;
        }
        __syncthreads();
    }
}


// ---- fused multi-request launch: frame layout -------------------------------------------------
//
// Two passes over units of kBatchChunk atoms of every packed frame, with the arithmetic of
// pack_count_kernel / pack_scatter_kernel: the count pass reads the staged positions and species
// (mapped host memory, all loads of a unit issued before any is used), copies them to device memory
// and counts species per unit; the scatter pass places each atom at its species offset (the plan's
// offsets plus the counts of the item's earlier units, stable within a unit by warp ranks), folds it
// and writes its fixed-point phase entry as well.
__global__ void __launch_bounds__(kBatchThreads) batch_count_kernel(const BatchHeader* __restrict__ hdr,
                                                                    const BatchItem* __restrict__ items,
                                                                    const float* __restrict__ xyz,
                                                                    const int32_t* __restrict__ sp,
                                                                    float4* __restrict__ raw,
                                                                    int32_t* __restrict__ chunk_counts,
                                                                    unsigned* status) {
    constexpr int kRounds = kBatchChunk / kBatchThreads;
    __shared__ int cnt[kBatchMaxSpecies];
    const int nitems = hdr->nitems;
    const int64_t total = hdr->total_chunk;
    for (int64_t u = blockIdx.x; u < total; u += gridDim.x) {
        const BatchItem& it = items[batch_item_of<&BatchItem::chunk_begin>(items, nitems, u)];
        const int64_t c = u - it.chunk_begin, off = it.atom_off;
        const int n = it.n, nsp = it.nsp;
        if (threadIdx.x < kBatchMaxSpecies) cnt[threadIdx.x] = 0;
        __syncthreads();
        float x[kRounds], y[kRounds], z[kRounds];
        int t[kRounds];
#pragma unroll
        for (int r = 0; r < kRounds; ++r) {
            const int64_t i = c * kBatchChunk + r * kBatchThreads + threadIdx.x;
            if (i < n) {
                x[r] = xyz[3 * (off + i)];
                y[r] = xyz[3 * (off + i) + 1];
                z[r] = xyz[3 * (off + i) + 2];
                t[r] = sp[off + i];
            }
        }
        bool bad = false;
#pragma unroll
        for (int r = 0; r < kRounds; ++r) {
            const int64_t i = c * kBatchChunk + r * kBatchThreads + threadIdx.x;
            if (i < n) {
                const bool ok = t[r] >= 0 && t[r] < nsp;
                if (!ok || !isfinite(x[r]) || !isfinite(y[r]) || !isfinite(z[r])) bad = true;
                if (ok) atomicAdd(&cnt[t[r]], 1);
                raw[off + i] = make_float4(x[r], y[r], z[r], __int_as_float(ok ? t[r] : -1));
            }
        }
        if (bad) trj_raise(status, TRJ_DEV_BAD_DATA);
        __syncthreads();
        if (threadIdx.x < kBatchMaxSpecies) chunk_counts[u * kBatchMaxSpecies + threadIdx.x] = cnt[threadIdx.x];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kBatchThreads) batch_scatter_kernel(const BatchHeader* __restrict__ hdr,
                                                                      const BatchItem* __restrict__ items,
                                                                      const float4* __restrict__ raw,
                                                                      const int32_t* __restrict__ chunk_counts,
                                                                      float4* __restrict__ packed,
                                                                      uint4* __restrict__ phase, unsigned* status) {
    constexpr int kRounds = kBatchChunk / kBatchThreads;
    __shared__ int64_t base[kBatchMaxSpecies];
    __shared__ int warp_cnt[kBatchThreads / 32][kBatchMaxSpecies];
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int nitems = hdr->nitems;
    const int64_t total = hdr->total_chunk;
    for (int64_t u = blockIdx.x; u < total; u += gridDim.x) {
        const BatchItem& it = items[batch_item_of<&BatchItem::chunk_begin>(items, nitems, u)];
        const int64_t c = u - it.chunk_begin, off = it.atom_off;
        const int n = it.n, nsp = it.nsp;
        const bool sorted = it.sp_off[nsp] >= 0;  // -1: g(r) only, atoms keep their order
        if (threadIdx.x < nsp) {
            int64_t b = it.sp_off[threadIdx.x];
            for (int64_t c2 = 0; c2 < c; ++c2) b += chunk_counts[(it.chunk_begin + c2) * kBatchMaxSpecies + threadIdx.x];
            base[threadIdx.x] = b;
        }
        for (int k = threadIdx.x; k < (kBatchThreads / 32) * kBatchMaxSpecies; k += kBatchThreads)
            (&warp_cnt[0][0])[k] = 0;
        __syncthreads();
        const double Lx = (double)it.L[0], Ly = (double)it.L[1], Lz = (double)it.L[2];
        for (int r = 0; r < kRounds; ++r) {
            const int64_t i = c * kBatchChunk + r * kBatchThreads + threadIdx.x;
            int s = -1;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (i < n) {
                v = raw[off + i];
                s = __float_as_int(v.w);  // -1 for a species flagged by the count pass: dropped
            }
            const unsigned peers = __match_any_sync(0xffffffffu, s);
            const int rank = __popc(peers & lt_mask);
            if (s >= 0 && rank == 0) warp_cnt[warp][s] = __popc(peers);
            __syncthreads();
            if (s >= 0) {
                int64_t pos = i;
                bool fits = true;
                if (sorted) {
                    pos = base[s] + rank;
                    for (int w = 0; w < warp; ++w) pos += warp_cnt[w][s];
                    fits = pos < it.sp_off[s + 1];  // more atoms of species s than the plan counts
                }
                if (fits) {
                    float4 f;
                    f.x = trj_fold_ref(v.x, it.L[0]);
                    f.y = trj_fold_ref(v.y, it.L[1]);
                    f.z = trj_fold_ref(v.z, it.L[2]);
                    f.w = __int_as_float(s);
                    packed[off + pos] = f;
                    phase[off + pos] = make_uint4(trj_phase_fraction(f.x, Lx), trj_phase_fraction(f.y, Ly),
                                                  trj_phase_fraction(f.z, Lz), (unsigned)s);
                } else {
                    trj_raise(status, TRJ_DEV_COUNT_MISMATCH);
                }
            } else if (!sorted && i < n) {
                packed[off + i] = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));  // no species: never paired
            }
            __syncthreads();
            if (threadIdx.x < nsp) {
                int tot = 0;
                for (int w = 0; w < kBatchThreads / 32; ++w) {
                    tot += warp_cnt[w][threadIdx.x];
                    warp_cnt[w][threadIdx.x] = 0;
                }
                base[threadIdx.x] += tot;
            }
            __syncthreads();
        }
        // the item's last unit: every species must have filled its range exactly
        if (sorted && c == it.nchunk - 1 && threadIdx.x < nsp && base[threadIdx.x] != it.sp_off[threadIdx.x + 1])
            trj_raise(status, TRJ_DEV_COUNT_MISMATCH);
        __syncthreads();
    }
}

}  // namespace

// Layout with context scratch; q/qpacked null for frames without charges.
static int frame_pack_impl(trj_ctx* ctx, const char* name, const float* xyz_dev, const int32_t* species_dev,
                           const float* charge_dev, int64_t n, int nsp, const float box[3], float* packed_dev,
                           float* charge_packed_dev, int64_t* counts_dev, void* stream,
                           const int32_t* lut_dev = nullptr, int nlut = 0) {
    if (!ctx) return TRJ_ERR_INVALID;
    if (n < 0 || nsp < 1 || nsp > kMaxSpecies || !box)
        return trj_fail(ctx, TRJ_ERR_INVALID, "%s: n=%lld nsp=%d (1..%d)", name, (long long)n, nsp, kMaxSpecies);
    if (!(box[0] > 0.f && box[1] > 0.f && box[2] > 0.f))
        return trj_fail(ctx, TRJ_ERR_INVALID, "%s: box edges must be positive", name);
    if (n > 0 && (!xyz_dev || !species_dev || !packed_dev))
        return trj_fail(ctx, TRJ_ERR_INVALID, "%s: null pointer", name);
    if (n > 0 && (charge_dev != nullptr) != (charge_packed_dev != nullptr))
        return trj_fail(ctx, TRJ_ERR_INVALID, "%s: charges need both the input and the output array", name);
    if (!counts_dev) return trj_fail(ctx, TRJ_ERR_INVALID, "%s: null counts", name);
    if (((uintptr_t)packed_dev) % 16 != 0)
        return trj_fail(ctx, TRJ_ERR_INVALID, "%s: packed_dev must be 16-byte aligned", name);
    trj_device_guard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    int64_t nblocks = (n + kPackChunk - 1) / kPackChunk;
    if (nblocks == 0) {
        TRJ_CUDA_TRY(ctx, cudaMemsetAsync(counts_dev, 0, sizeof(int64_t) * nsp, s));
        return TRJ_OK;
    }
    if (nblocks > (int64_t)INT32_MAX) return trj_fail(ctx, TRJ_ERR_INVALID, "frame too large");
    size_t need = (size_t)nblocks * nsp * (sizeof(int32_t) + sizeof(int64_t)) + 256;
    trj_ctx::PackScratch& ps = ctx->pack_scratch[stream];
    if (need > ps.bytes) {
        // Earlier layout kernels of this stream may still use the old buffer, and neither cudaFree's
        // implicit synchronisation nor a caller's free callback (which takes no stream) orders the
        // release after them: wait for the stream first.
        if (ps.ptr) TRJ_CUDA_TRY(ctx, cudaStreamSynchronize(s));
        trj_dev_free(ctx, ps.ptr);
        ps.ptr = nullptr;
        ps.bytes = 0;
        if (trj_dev_alloc(ctx, &ps.ptr, need) != cudaSuccess)
            return trj_fail(ctx, TRJ_ERR_NOMEM, "%s: scratch of %zu bytes", name, need);
        ps.bytes = need;
    }
    int64_t* block_base = (int64_t*)ps.ptr;
    int32_t* block_counts = (int32_t*)(block_base + nblocks * nsp);
    pack_count_kernel<<<(unsigned)nblocks, kPackThreads, 0, s>>>(xyz_dev, species_dev, n, nsp,
                                                                 block_counts, ctx->status_dev, lut_dev, nlut);
    pack_scan_kernel<<<1, 1024, 0, s>>>(block_counts, nblocks, nsp, counts_dev, block_base);
    pack_scatter_kernel<<<(unsigned)nblocks, kPackThreads, 0, s>>>(xyz_dev, species_dev, n, nsp, box[0], box[1],
                                                                   box[2], block_base, (float4*)packed_dev,
                                                                   charge_dev, charge_packed_dev, lut_dev, nlut);
    ctx->launches += 3;
    TRJ_CUDA_TRY(ctx, cudaGetLastError());
    return TRJ_OK;
}

extern "C" int trj_frame_pack(trj_ctx* ctx, const float* xyz_dev, const int32_t* species_dev,
                              int64_t n, int nsp, const float box[3], float* packed_dev,
                              int64_t* counts_dev, void* stream) {
    return frame_pack_impl(ctx, "trj_frame_pack", xyz_dev, species_dev, nullptr, n, nsp, box, packed_dev, nullptr,
                           counts_dev, stream);
}

extern "C" int trj_frame_pack_types(trj_ctx* ctx, const float* xyz_dev, const int32_t* types_dev,
                                    const int32_t* lut_dev, int nlut, int64_t n, int nsp, const float box[3],
                                    float* packed_dev, int64_t* counts_dev, void* stream) {
    if (ctx && (!lut_dev || nlut < 1))
        return trj_fail(ctx, TRJ_ERR_INVALID, "trj_frame_pack_types: null or empty type table");
    return frame_pack_impl(ctx, "trj_frame_pack_types", xyz_dev, types_dev, nullptr, n, nsp, box, packed_dev, nullptr,
                           counts_dev, stream, lut_dev, nlut);
}

extern "C" int trj_frame_pack_charges(trj_ctx* ctx, const float* xyz_dev, const int32_t* species_dev,
                                      const float* charge_dev, int64_t n, int nsp, const float box[3],
                                      float* packed_dev, float* charge_packed_dev, int64_t* counts_dev,
                                      void* stream) {
    if (ctx && n > 0 && (!charge_dev || !charge_packed_dev))
        return trj_fail(ctx, TRJ_ERR_INVALID, "trj_frame_pack_charges: null charge array");
    return frame_pack_impl(ctx, "trj_frame_pack_charges", xyz_dev, species_dev, charge_dev, n, nsp, box, packed_dev,
                           charge_packed_dev, counts_dev, stream);
}

// ---------------------------------------------------------------------------
// Frame layout without allocation.
//
// trj_frame_pack_static runs the same three layout kernels as trj_frame_pack, but its
// per-block species counts and block offsets live in the fixed device array below instead of
// context scratch grown with cudaMalloc.  It serves callers that may not allocate device memory
// from inside the library: applications whose device memory is owned by another allocator (a
// framework's caching allocator, a pre-sized arena) and that forbid foreign allocations, and
// frame loops that cannot take the implicit device synchronisation of cudaMalloc/cudaFree.
//
// Limit: ceil(n / 1024) * nsp * 12 bytes must fit in kPackStaticBytes (1 MiB), i.e.
// ceil(n / 1024) * nsp <= 87381 (about 29.8 million atoms for 3 species, 5.5 million for 16).
// Every GPU that loads this library holds the 1 MiB array until the process exits.  The array's
// address is resolved once per device and kept for the life of the process, so resetting a device
// (cudaDeviceReset) after the first call on it is not supported.  All calls
// share it: each call overwrites every word it reads (nothing has to start at zero), and calls
// whose kernels overlap on the GPU (different streams, other host threads) race on it.
// ---------------------------------------------------------------------------

constexpr size_t kPackStaticBytes = (size_t)1 << 20;
static __device__ __align__(256) unsigned char g_pack_static[kPackStaticBytes];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_pack_static_mu;
void* g_pack_static_addr[kMaxDevices] = {};

// Device address of g_pack_static on the current device, resolved once per device.
int pack_static_address(trj_ctx* ctx, void** out) {
    if (ctx->device < 0 || ctx->device >= kMaxDevices)
        return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "trj_frame_pack_static: device ordinal %d >= %d", ctx->device,
                        kMaxDevices);
    std::lock_guard<std::mutex> lock(g_pack_static_mu);
    if (!g_pack_static_addr[ctx->device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_pack_static);
        if (e != cudaSuccess || !p)
            return trj_fail(ctx, TRJ_ERR_CUDA, "trj_frame_pack_static: cudaGetSymbolAddress failed: %s",
                            cudaGetErrorString(e));
        g_pack_static_addr[ctx->device] = p;
    }
    *out = g_pack_static_addr[ctx->device];
    return TRJ_OK;
}
}  // namespace

extern "C" int trj_frame_pack_static(trj_ctx* ctx, const float* xyz_dev, const int32_t* species_dev, int64_t n,
                                     int nsp, const float box[3], float* packed_dev, int64_t* counts_dev,
                                     void* stream) {
    if (!ctx) return TRJ_ERR_INVALID;
    if (n < 0 || nsp < 1 || nsp > kMaxSpecies || !box)
        return trj_fail(ctx, TRJ_ERR_INVALID, "trj_frame_pack_static: n=%lld nsp=%d (1..%d)", (long long)n, nsp,
                        kMaxSpecies);
    if (!(box[0] > 0.f && box[1] > 0.f && box[2] > 0.f))
        return trj_fail(ctx, TRJ_ERR_INVALID, "trj_frame_pack_static: box edges must be positive");
    if (n > 0 && (!xyz_dev || !species_dev || !packed_dev))
        return trj_fail(ctx, TRJ_ERR_INVALID, "trj_frame_pack_static: null pointer");
    if (!counts_dev) return trj_fail(ctx, TRJ_ERR_INVALID, "trj_frame_pack_static: null counts");
    if (((uintptr_t)packed_dev) % 16 != 0)
        return trj_fail(ctx, TRJ_ERR_INVALID, "trj_frame_pack_static: packed_dev must be 16-byte aligned");
    const int64_t nblocks = (n + kPackChunk - 1) / kPackChunk;
    const size_t need = (size_t)nblocks * nsp * (sizeof(int64_t) + sizeof(int32_t));
    if (need > kPackStaticBytes)
        return trj_fail(ctx, TRJ_ERR_CAPACITY,
                        "trj_frame_pack_static: n=%lld with nsp=%d needs %zu bytes of scratch; the fixed array holds "
                        "%zu (ceil(n/1024)*nsp must be <= %zu)",
                        (long long)n, nsp, need, kPackStaticBytes, kPackStaticBytes / 12);
    trj_device_guard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    if (nblocks == 0) {
        TRJ_CUDA_TRY(ctx, cudaMemsetAsync(counts_dev, 0, sizeof(int64_t) * nsp, s));
        return TRJ_OK;
    }
    void* scratch = nullptr;
    int rc = pack_static_address(ctx, &scratch);
    if (rc != TRJ_OK) return rc;
    int64_t* block_base = (int64_t*)scratch;
    int32_t* block_counts = (int32_t*)(block_base + nblocks * nsp);
    pack_count_kernel<<<(unsigned)nblocks, kPackThreads, 0, s>>>(xyz_dev, species_dev, n, nsp, block_counts,
                                                                 ctx->status_dev, nullptr, 0);
    pack_scan_kernel<<<1, 1024, 0, s>>>(block_counts, nblocks, nsp, counts_dev, block_base);
    pack_scatter_kernel<<<(unsigned)nblocks, kPackThreads, 0, s>>>(xyz_dev, species_dev, n, nsp, box[0], box[1],
                                                                   box[2], block_base, (float4*)packed_dev, nullptr,
                                                                   nullptr, nullptr, 0);
    ctx->launches += 3;
    TRJ_CUDA_TRY(ctx, cudaGetLastError());
    return TRJ_OK;
}

void trj_batch_launch_layout(const BatchHeader* hdr, const BatchItem* items, const float* xyz_staged,
                             const int32_t* sp_staged, float4* raw, int32_t* chunk_counts, float4* packed,
                             uint4* phase, unsigned* status, int grid, cudaStream_t s) {
    batch_count_kernel<<<grid, kBatchThreads, 0, s>>>(hdr, items, xyz_staged, sp_staged, raw, chunk_counts, status);
    batch_scatter_kernel<<<grid, kBatchThreads, 0, s>>>(hdr, items, raw, chunk_counts, packed, phase, status);
}
