// batch.cuh -- descriptors of the fused multi-request launches (trj_batch_*).
//
// A turn packs one frame of each of up to max_items small requests.  The host writes the frames'
// positions and species ids back to back into mapped pinned staging and one BatchItem per frame into
// a pinned table; the launch sequence (table copy, layout count, layout scatter, pair histogram,
// direct sum, shell reduction) is the same for every turn, so one CUDA graph per staging buffer
// replays any mix of requests.  Every kernel walks a global list of work units; an item's units
// start at its *_begin offset (exclusive prefix over the items before it).
#pragma once

#include "trj_common.cuh"

constexpr int kBatchChunk = 1024;        // atoms per layout unit
constexpr int kBatchTile = 256;          // atoms per side of a pair tile (one home atom per thread)
constexpr int kBatchThreads = 256;
constexpr int kBatchMaxSpecies = 16;
constexpr int kBatchCounters = 4;        // dynamic work counters: pairs, direct sum, reduction, spare

struct __align__(16) BatchItem {
    // frame: atoms [atom_off, atom_off + n) of the staging and device arrays
    int64_t atom_off;
    int32_t n, nsp;
    float L[3];
    int32_t nchunk;                      // layout units: ceil(n / kBatchChunk)
    int32_t ntile;                       // pair tiles per side: ceil(n / kBatchTile)
    int32_t nit;
    int64_t sp_off[kBatchMaxSpecies + 1];  // species offsets of the S(Q) plan within the frame
    // pair histogram (the rdf plan's geometry after the per-frame clip)
    float h1[3], h2[3], pad_h[3];        // minimum-image thresholds (rdf.cu min_image)
    float side2, side2_lo, side2_hi, deltar, inv_deltar;
    int32_t lsmax, floor_bins;
    unsigned long long* hist;            // [nit][lsmax] accumulator
    unsigned long long* edge;            // edge counters (ulp, fma, counted) or null
    // S(Q) direct sum over the plan's vectors (the plain method of trj_sq_accumulate)
    const int4* vecs;
    const int32_t* subset;
    const double* w;
    const int32_t* bin_start;
    const int64_t* sp_off_dev;
    double2* part;                       // [nsplit][nsp][nvec]
    double2* rho;                        // [nsp][nvec]
    double* out;                         // [nbins][nit] accumulator
    int32_t nvec, nsplit, vpt, nbins;
    int32_t nvblk;                       // vector blocks: ceil(nvec / (kBatchThreads * vpt))
    int32_t pad0;
    // first work unit of the item in each kernel's list
    int64_t chunk_begin, pair_begin, sq_begin, red_begin;
};

struct __align__(16) BatchHeader {
    unsigned long long counter[kBatchCounters];  // zero in every turn's copy of the table
    int32_t nitems, pad0;
    int64_t total_chunk, total_pair, total_sq, total_red, total_atoms;
    int64_t pad1[2];
};
static_assert(sizeof(BatchHeader) % 16 == 0, "table alignment");
static_assert(sizeof(BatchItem) % 16 == 0, "table alignment");

// Item of work unit u: the last item whose begin offset (member `field` of BatchItem) is <= u.
template <int64_t BatchItem::*field>
__device__ __forceinline__ int batch_item_of(const BatchItem* __restrict__ items, int nitems, int64_t u) {
    int lo = 0, hi = nitems - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].*field <= u) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Kernel launchers of the fused turn, each defined beside the single-request kernels whose
// arithmetic it shares.  grid: CTAs of the fixed-size launch.
void trj_batch_launch_layout(const BatchHeader* hdr, const BatchItem* items, const float* xyz_staged,
                             const int32_t* sp_staged, float4* raw, int32_t* chunk_counts, float4* packed,
                             uint4* phase, unsigned* status, int grid, cudaStream_t s);        // ctx.cu
void trj_batch_launch_pairs(BatchHeader* hdr, const BatchItem* items, const float4* packed, int hist_words,
                            int grid, cudaStream_t s);                                        // rdf.cu
size_t trj_batch_pairs_smem(int hist_words);                                                  // rdf.cu
int trj_batch_pairs_prepare(int hist_words);                                                  // rdf.cu
int trj_batch_pairs_occupancy(int hist_words, int* per_sm);                                   // rdf.cu
void trj_batch_launch_sq(BatchHeader* hdr, const BatchItem* items, const uint4* phase, int grid_sq, int grid_red,
                         cudaStream_t s);                                                     // sq.cu
int trj_batch_sq_occupancy(int* per_sm_sq, int* per_sm_red);                                   // sq.cu
struct trj_rdf_plan;
struct trj_sq_plan;
// Fill the pair part of an item from a plan after the per-frame clip (rdf.cu), and the S(Q) part
// (sq.cu); non-zero: the plan cannot run in a fused launch (the message is on the context).
int trj_batch_fill_rdf(trj_rdf_plan* plan, const float box[3], int hist_words, BatchItem* it, int* nsp);
int trj_batch_fill_sq(trj_sq_plan* plan, int64_t n, BatchItem* it);
