// batch.cu -- fused multi-request launches: one frame of each of several small requests per turn.
//
// The reference analyses one trajectory per process and one frame per step of its main loop
// (src/main/trj_analysis.f90:208-217: transfer_cpu_gpu, RDFcomp, SQcalc, each a fixed-shape launch
// over that frame, rdf.cuf:240 and sq.cuf:89).  A serving loop with many small requests would pay
// those launches per request and frame.  A batch instead takes one frame of every packed request per
// turn and runs the same fixed sequence of launches for all of them:
//
//   copy of the pinned descriptor table -> layout count -> layout scatter (fold, species order,
//   fixed-point phases) -> all-pairs histogram -> direct sum -> shell reduction
//
// Grids and arguments depend only on the batch's capacity, so a CUDA graph captured once per staging
// buffer replays any mix of requests: the host rewrites the table and the staged atoms between turns.
#include <algorithm>

#include "batch.cuh"
#include "sq_plan.cuh"

struct trj_batch {
    trj_ctx* ctx = nullptr;
    int max_items = 0;
    int64_t max_atoms = 0;
    int hist_words = 0;
    int grid_layout = 0, grid_pairs = 0, grid_sq = 0, grid_red = 0;
    size_t table_bytes = 0;
    int64_t device_bytes = 0;
    struct Buf {
        unsigned char* table_host = nullptr;  // pinned: BatchHeader + max_items BatchItems
        unsigned char* table_dev = nullptr;
        float* xyz_host = nullptr;            // mapped pinned staging: 3 floats per atom
        int32_t* sp_host = nullptr;           // mapped pinned staging: species id per atom
        float* xyz_map = nullptr;             // device addresses of the same
        int32_t* sp_map = nullptr;
        float4* raw = nullptr;                // device: staged atoms before the layout
        float4* packed = nullptr;             // device: folded atoms in species order
        uint4* phase = nullptr;               // device: fixed-point phase entries
        int32_t* chunk_counts = nullptr;      // device: species counts per layout unit
        int64_t atoms_end = 0;                // end of the last item's atoms
        int64_t chunk_cap = 0;
        BatchHeader* hdr() { return reinterpret_cast<BatchHeader*>(table_host); }
        BatchItem* items() { return reinterpret_cast<BatchItem*>(table_host + sizeof(BatchHeader)); }
    } buf[2];
    trj_kernel_timer timer;
};

static void batch_free(trj_batch* b) {
    trj_device_guard g(b->ctx->device);
    for (auto& B : b->buf) {
        if (B.table_host) cudaFreeHost(B.table_host);
        if (B.xyz_host) cudaFreeHost(B.xyz_host);
        if (B.sp_host) cudaFreeHost(B.sp_host);
        trj_dev_free(b->ctx, B.table_dev);
        B = trj_batch::Buf();
    }
    b->timer.release();
}

extern "C" int trj_batch_create(trj_ctx* ctx, int max_items, int64_t max_atoms, int hist_words, trj_batch** out) {
    if (!ctx || !out) return TRJ_ERR_INVALID;
    *out = nullptr;
    if (max_items < 1 || max_items > 4096 || max_atoms < 1 || max_atoms > ((int64_t)1 << 31) || hist_words < 1 ||
        hist_words > 24576)
        return trj_fail(ctx, TRJ_ERR_INVALID, "batch: max_items=%d (1..4096), max_atoms=%lld (1..2^31), "
                        "hist_words=%d (1..24576)", max_items, (long long)max_atoms, hist_words);
    trj_device_guard g(ctx->device);
    trj_batch* b = new trj_batch();
    b->ctx = ctx;
    b->max_items = max_items;
    b->max_atoms = max_atoms;
    b->hist_words = hist_words;
    b->table_bytes = sizeof(BatchHeader) + (size_t)max_items * sizeof(BatchItem);
    auto a256 = [](size_t x) { return (x + 255) & ~(size_t)255; };
    for (auto& B : b->buf) {
        B.chunk_cap = (max_atoms + kBatchChunk - 1) / kBatchChunk + max_items;
        const size_t dev = a256(b->table_bytes) + 3 * a256(sizeof(float4) * (size_t)max_atoms) +
                           a256(sizeof(int32_t) * kBatchMaxSpecies * (size_t)B.chunk_cap);
        if (cudaHostAlloc((void**)&B.table_host, b->table_bytes, cudaHostAllocDefault) != cudaSuccess ||
            cudaHostAlloc((void**)&B.xyz_host, sizeof(float) * 3 * (size_t)max_atoms,
                          cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess ||
            cudaHostAlloc((void**)&B.sp_host, sizeof(int32_t) * (size_t)max_atoms,
                          cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess ||
            cudaHostGetDevicePointer((void**)&B.xyz_map, B.xyz_host, 0) != cudaSuccess ||
            cudaHostGetDevicePointer((void**)&B.sp_map, B.sp_host, 0) != cudaSuccess) {
            cudaGetLastError();
            batch_free(b);
            delete b;
            return trj_fail(ctx, TRJ_ERR_NOMEM, "batch: pinned staging for %lld atoms", (long long)max_atoms);
        }
        if (trj_dev_alloc(ctx, (void**)&B.table_dev, dev) != cudaSuccess) {
            batch_free(b);
            delete b;
            return trj_fail(ctx, TRJ_ERR_NOMEM, "batch: %zu bytes of device memory", dev);
        }
        unsigned char* p = B.table_dev + a256(b->table_bytes);
        B.raw = reinterpret_cast<float4*>(p);
        p += a256(sizeof(float4) * (size_t)max_atoms);
        B.packed = reinterpret_cast<float4*>(p);
        p += a256(sizeof(float4) * (size_t)max_atoms);
        B.phase = reinterpret_cast<uint4*>(p);
        p += a256(sizeof(float4) * (size_t)max_atoms);
        B.chunk_counts = reinterpret_cast<int32_t*>(p);
        b->device_bytes += (int64_t)dev;
        memset(B.table_host, 0, b->table_bytes);
    }
    if (trj_batch_pairs_prepare(hist_words) != 0) {
        batch_free(b);
        delete b;
        return trj_fail(ctx, TRJ_ERR_UNSUPPORTED, "batch: %zu bytes of shared memory for the pair kernel",
                        trj_batch_pairs_smem(hist_words));
    }
    int occ_pairs = 0, occ_sq = 0, occ_red = 0;
    if (trj_batch_pairs_occupancy(hist_words, &occ_pairs) != 0 || trj_batch_sq_occupancy(&occ_sq, &occ_red) != 0) {
        batch_free(b);
        delete b;
        return trj_fail(ctx, TRJ_ERR_CUDA, "batch: occupancy query failed");
    }
    b->grid_layout = ctx->sm_count * 4;
    b->grid_pairs = ctx->sm_count * occ_pairs;
    b->grid_sq = ctx->sm_count * std::max(1, occ_sq);
    b->grid_red = ctx->sm_count * std::max(1, occ_red);
    *out = b;
    return TRJ_OK;
}

extern "C" int trj_batch_destroy(trj_batch* b) {
    if (!b) return TRJ_OK;
    {
        trj_device_guard g(b->ctx->device);
        cudaDeviceSynchronize();  // pinned staging may still feed a launch of the caller's stream
    }
    batch_free(b);
    delete b;
    return TRJ_OK;
}

extern "C" int trj_batch_staging(trj_batch* b, int buf, float** xyz_host, int32_t** species_host) {
    if (!b) return TRJ_ERR_INVALID;
    if (buf < 0 || buf > 1) return trj_fail(b->ctx, TRJ_ERR_INVALID, "batch: staging buffer %d (0 or 1)", buf);
    if (xyz_host) *xyz_host = b->buf[buf].xyz_host;
    if (species_host) *species_host = b->buf[buf].sp_host;
    return TRJ_OK;
}

extern "C" int trj_batch_begin(trj_batch* b, int buf) {
    if (!b) return TRJ_ERR_INVALID;
    if (buf < 0 || buf > 1) return trj_fail(b->ctx, TRJ_ERR_INVALID, "batch: staging buffer %d (0 or 1)", buf);
    auto& B = b->buf[buf];
    memset(B.hdr(), 0, sizeof(BatchHeader));
    B.atoms_end = 0;
    return TRJ_OK;
}

extern "C" int trj_batch_add(trj_batch* b, int buf, trj_rdf_plan* rdf, trj_sq_plan* sq, int64_t atom_off, int64_t n,
                             const float box[3], uint64_t* hist_dev, uint64_t* edge_dev, double* sq_out_dev) {
    if (!b) return TRJ_ERR_INVALID;
    trj_ctx* ctx = b->ctx;
    if (buf < 0 || buf > 1) return trj_fail(ctx, TRJ_ERR_INVALID, "batch: staging buffer %d (0 or 1)", buf);
    auto& B = b->buf[buf];
    BatchHeader* h = B.hdr();
    if (h->nitems >= b->max_items) return trj_fail(ctx, TRJ_ERR_CAPACITY, "batch: %d items already", h->nitems);
    if (!rdf && !sq) return trj_fail(ctx, TRJ_ERR_INVALID, "batch: an item needs a pair plan, an S(Q) plan or both");
    if (!box || !(box[0] > 0.f && box[1] > 0.f && box[2] > 0.f))
        return trj_fail(ctx, TRJ_ERR_INVALID, "batch: box edges must be positive");
    if (n < 0 || n > INT32_MAX || atom_off < B.atoms_end || atom_off + n > b->max_atoms)
        return trj_fail(ctx, TRJ_ERR_CAPACITY, "batch: atoms [%lld, %lld) outside [%lld, %lld) (items in atom order)",
                        (long long)atom_off, (long long)(atom_off + n), (long long)B.atoms_end,
                        (long long)b->max_atoms);
    if ((rdf && !hist_dev) || (sq && !sq_out_dev))
        return trj_fail(ctx, TRJ_ERR_INVALID, "batch: null accumulator");
    BatchItem it;
    memset(&it, 0, sizeof(it));
    it.atom_off = atom_off;
    it.n = (int32_t)n;
    for (int d = 0; d < 3; ++d) it.L[d] = box[d];
    for (int a = 0; a <= kBatchMaxSpecies; ++a) it.sp_off[a] = -1;  // g(r) only: atoms keep their order
    int nsp = 0;
    if (sq) {
        int rc = trj_batch_fill_sq(sq, n, &it);
        if (rc != TRJ_OK) return rc;
        it.out = sq_out_dev;
        nsp = sq->nsp;
    }
    if (rdf) {
        int p_nsp = 0;
        int rc = trj_batch_fill_rdf(rdf, box, b->hist_words, &it, &p_nsp);
        if (rc != TRJ_OK) return rc;
        if (sq && p_nsp != nsp)
            return trj_fail(ctx, TRJ_ERR_INVALID, "batch: pair plan has %d species, S(Q) plan %d", p_nsp, nsp);
        nsp = p_nsp;
        it.hist = (unsigned long long*)hist_dev;
        it.edge = (unsigned long long*)edge_dev;
    }
    it.nsp = nsp;
    it.nchunk = (int32_t)((n + kBatchChunk - 1) / kBatchChunk);
    it.ntile = rdf && n >= 2 ? (int32_t)((n + kBatchTile - 1) / kBatchTile) : 0;
    it.chunk_begin = h->total_chunk;
    it.pair_begin = h->total_pair;
    it.sq_begin = h->total_sq;
    it.red_begin = h->total_red;
    if (h->total_chunk + it.nchunk > B.chunk_cap)
        return trj_fail(ctx, TRJ_ERR_CAPACITY, "batch: layout units exceed %lld", (long long)B.chunk_cap);
    h->total_chunk += it.nchunk;
    h->total_pair += (int64_t)it.ntile * (it.ntile + 1) / 2;
    if (sq && it.nvec > 0) {
        h->total_sq += (int64_t)it.nvblk * it.nsplit;
        h->total_red += it.nbins;
    }
    h->total_atoms += n;
    B.items()[h->nitems] = it;
    h->nitems += 1;
    B.atoms_end = atom_off + n;
    return TRJ_OK;
}

extern "C" int trj_batch_launch(trj_batch* b, int buf, void* stream) {
    if (!b) return TRJ_ERR_INVALID;
    trj_ctx* ctx = b->ctx;
    if (buf < 0 || buf > 1) return trj_fail(ctx, TRJ_ERR_INVALID, "batch: staging buffer %d (0 or 1)", buf);
    trj_device_guard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    auto& B = b->buf[buf];
    BatchHeader* hdr = reinterpret_cast<BatchHeader*>(B.table_dev);
    const BatchItem* items = reinterpret_cast<const BatchItem*>(B.table_dev + sizeof(BatchHeader));
    // The same launches whatever the table holds (a captured graph replays them): the copy reads
    // the pinned table when it executes.
    TRJ_CUDA_TRY(ctx, cudaMemcpyAsync(B.table_dev, B.table_host, b->table_bytes, cudaMemcpyHostToDevice, s));
    b->timer.begin(ctx, s);
    trj_batch_launch_layout(hdr, items, B.xyz_map, B.sp_map, B.raw, B.chunk_counts, B.packed, B.phase,
                            ctx->status_dev, b->grid_layout, s);
    trj_batch_launch_pairs(hdr, items, B.packed, b->hist_words, b->grid_pairs, s);
    trj_batch_launch_sq(hdr, items, B.phase, b->grid_sq, b->grid_red, s);
    b->timer.end(ctx, s);
    ctx->launches += 5;
    TRJ_CUDA_TRY(ctx, cudaGetLastError());
    return TRJ_OK;
}

extern "C" int trj_batch_info(const trj_batch* b, int buf, int* nitems, int64_t units[4], int64_t* device_bytes) {
    if (!b || buf < 0 || buf > 1) return TRJ_ERR_INVALID;
    const BatchHeader* h = reinterpret_cast<const BatchHeader*>(b->buf[buf].table_host);
    if (nitems) *nitems = h->nitems;
    if (units) {
        units[0] = h->total_chunk;
        units[1] = h->total_pair;
        units[2] = h->total_sq;
        units[3] = h->total_red;
    }
    if (device_bytes) *device_bytes = b->device_bytes;
    return TRJ_OK;
}

extern "C" int trj_batch_kernel_ms(trj_batch* b, float* ms) {
    if (!b) return TRJ_ERR_INVALID;
    return b->timer.elapsed(b->ctx, ms);
}
