// sq_plan.cuh -- S(Q) plan layout shared by the direct-sum and tensor-core kernels.
#pragma once
#include <vector>

#include "trj_common.cuh"

// Tensor-core tile geometry: 128 rows = 16 nx values x 8 ny values; columns are
// (nz, re/im) pairs, 2*nz_count columns padded to a multiple of 16 (<= 224).
constexpr int kTcTileNx = 16;
constexpr int kTcTileNy = 8;
constexpr int kTcRows = kTcTileNx * kTcTileNy;  // 128
constexpr int kTcMaxCols = 224;

struct SqTile {
    int nx0, ny0, nz0;  // lattice origin of the tile
    int ncols;          // output columns = 2 * nz span, padded to 16
    int64_t out_off;    // offset (in doubles) of this tile's FP64 rho block: [nsp][ncols][128]
};

struct trj_sq_plan {
    trj_ctx* ctx = nullptr;
    int nsp = 0, nit = 0, nbins = 0;
    int64_t nvec = 0;
    int64_t n_total = 0;                   // phase entries: atoms, plus the charge species' copies
    int64_t n_atoms = 0;                   // atoms per frame
    int qsp = -1;                          // index of the charge species (charged plans), else -1
    unsigned z_from_y = 0;                 // planar tile form: third phase = z_from_y * u_y (0: off)
    std::vector<int64_t> species_counts;   // host
    std::vector<int64_t> species_off;      // host, nsp+1
    // vectors in plan order (sorted by bin); perm[plan_index] = caller index
    int4* vec_dev = nullptr;               // nx, ny, nz, caller index
    double* weight_dev = nullptr;
    int32_t* bin_start_dev = nullptr;      // nbins + 1
    int64_t* species_off_dev = nullptr;    // nsp + 1
    // direct-sum subsets (plan-order indices)
    int32_t* plain_all_dev = nullptr;      // every vector (plain method)
    int32_t* plain_sparse_dev = nullptr;   // non-dense vectors (tensor method)
    int64_t n_sparse = 0;
    // tensor-core tiles
    std::vector<SqTile> tiles;
    SqTile* tiles_dev = nullptr;
    int64_t n_dense = 0;
    int64_t tile_slots = 0;                // sum over tiles of 128 * ncols/2
    int64_t tc_out_doubles = 0;
    int64_t* dense_src_dev = nullptr;      // per plan vector: offset into TC output (re at +0, im at +128) or -1
    // scratch
    uint4* phase_dev = nullptr;            // n_total x (ux, uy, uz, species)
    double2* part_dev = nullptr;           // direct-sum partials [nsplit][nsp][nvec]
    int nsplit_all = 1, nsplit_sparse = 1;
    double* tc_out_dev = nullptr;          // tensor-core rho blocks (FP64)
    double2* rho_dev = nullptr;            // [nsp][nvec] final rho in plan order
    int last_method = -1;
    int64_t scratch_bytes = 0;
    void* tc_state = nullptr;              // tensor-core kernel private state
    void* groups_buf = nullptr;            // scratch of trj_sq_rho_groups (grown on demand)
    size_t groups_bytes = 0;
    trj_kernel_timer timer;                // around the main kernel of the last accumulate
};

// Tensor-core path entry (sq_tc.cu).  Computes FP64 rho blocks of all tiles into
// plan->tc_out_dev from plan->phase_dev.
int trj_sq_tc_run(trj_sq_plan* plan, const float box[3], cudaStream_t s);
int trj_sq_tc_prepare(trj_sq_plan* plan);
void trj_sq_tc_release(trj_sq_plan* plan);
