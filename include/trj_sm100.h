/*
 * trj_sm100.h -- C ABI of the B200 (sm_100a) g_ab(r) / S_ab(Q) library.
 *
 * Plain C: pointers, sizes and status codes only.  Every call returns an int
 * status (TRJ_OK == 0, negative on error) and never exits the process; the
 * message of the last error of a context is read with trj_ctx_last_error().
 * Device pointers are CUDA global-memory addresses on the context's device.
 * `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 * Calls are asynchronous on `stream` unless stated otherwise; device-side
 * status (bad input data, bounded-wait timeouts) is collected by
 * trj_ctx_check(), which synchronises the stream.
 *
 * The reference implements this path as Fortran subroutines that read module
 * globals (CUDA Fortran, src/modules/rdf.cuf and src/modules/sq.cuf).  Each
 * entry point below names the reference routine whose role it takes.
 * Threading: a context and its plans may be used from one host thread at a
 * time (use one context per thread).  Work of one context may run on several
 * streams at once: frame-layout scratch is kept per stream, plans own theirs
 * (one plan must not run on two streams at the same time).
 */
#ifndef TRJ_SM100_H
#define TRJ_SM100_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TRJ_ABI_VERSION 1

#if defined(__GNUC__)
#define TRJ_API __attribute__((visibility("default")))
#else
#define TRJ_API
#endif

/* status codes */
#define TRJ_OK               0
#define TRJ_ERR_INVALID     -1   /* bad argument (shape, range, null pointer)          */
#define TRJ_ERR_CUDA        -2   /* a CUDA runtime call failed                         */
#define TRJ_ERR_NOMEM       -3   /* device or host allocation failed                  */
#define TRJ_ERR_CAPACITY    -4   /* input larger than the plan was sized for          */
#define TRJ_ERR_DATA        -5   /* non-finite positions or species out of range      */
#define TRJ_ERR_UNSUPPORTED -6   /* configuration not supported by this build/device  */
#define TRJ_ERR_TIMEOUT     -7   /* a bounded device-side wait ran out                */

/* S(Q) methods */
#define TRJ_SQ_PLAIN_FP32    0   /* direct sum, one phase per atom and k-vector (CUDA cores) */
#define TRJ_SQ_SPLIT_BF16X3  1   /* separable phases, tcgen05 BF16 hi/lo 3-term contraction  */

typedef struct trj_ctx trj_ctx;
typedef struct trj_rdf_plan trj_rdf_plan;
typedef struct trj_sq_plan trj_sq_plan;
typedef struct trj_dyn_plan trj_dyn_plan;
typedef struct trj_batch trj_batch;

/* Edge-pair statistics of one or more accumulate calls (device uint64[4]). */
enum {
    TRJ_EDGE_ULP = 0,      /* pairs whose outcome changes when rr2 moves one FP32 ulp */
    TRJ_EDGE_FMA = 1,      /* pairs whose outcome changes under the FMA-contracted rr2 */
    TRJ_EDGE_COUNTED = 2,  /* pairs counted into the histogram                       */
    TRJ_EDGE_TESTED = 3    /* candidate pairs tested (cell-list work)                */
};

TRJ_API int trj_abi_version(void);

/* ---- context --------------------------------------------------------- */
/* Replaces the device selection and module set-up of gpu_and_header
 * (src/core/util.f90:54-80) and common_init (src/core/common.cuf:380-468). */
TRJ_API int trj_ctx_create(int device, trj_ctx** out);
TRJ_API int trj_ctx_destroy(trj_ctx* ctx);
TRJ_API const char* trj_ctx_last_error(const trj_ctx* ctx);
/* Synchronise `stream` and report device-side status raised since the last check
 * (TRJ_ERR_DATA / TRJ_ERR_TIMEOUT / TRJ_ERR_CAPACITY), then clear it. */
TRJ_API int trj_ctx_check(trj_ctx* ctx, void* stream);
TRJ_API int trj_ctx_sm_count(const trj_ctx* ctx);
/* Device memory of plans and scratch.  By default the library calls cudaMalloc
 * and cudaFree (and cudaFree synchronises the device).  A caller that owns
 * device memory through its own allocator (for example a caching allocator, so
 * that plans can be created and destroyed while other streams keep running)
 * installs alloc/free callbacks here: alloc(bytes, user) returns a device
 * pointer (256-byte aligned) or NULL; free(ptr, user) releases it.  Install
 * them right after trj_ctx_create, before any plan exists; pass NULLs to return
 * to cudaMalloc/cudaFree.  The callbacks are called from the thread that
 * creates or destroys a plan. */
typedef void* (*trj_alloc_fn)(size_t bytes, void* user);
typedef void (*trj_free_fn)(void* ptr, void* user);
TRJ_API int trj_ctx_set_allocator(trj_ctx* ctx, trj_alloc_fn alloc, trj_free_fn free_fn, void* user);
/* Kernel timing: when enabled, each accumulate call records CUDA events on its
 * stream around the plan's main kernel (the cell-pair kernel, the tcgen05 S(Q)
 * kernel, or the direct-sum kernel); trj_*_kernel_ms reads the last duration
 * (synchronises on the stop event).  Off by default. */
TRJ_API int trj_ctx_set_timing(trj_ctx* ctx, int enable);
/* Number of kernels this library has launched on the context so far. */
TRJ_API int64_t trj_ctx_launches(const trj_ctx* ctx);
/* Widest tensor-core S(Q) tile (output columns: 2 per nz value) of the S(Q)
 * plans this context creates from now on: 0 (default, 224) or 32..224 in steps
 * of 16.  Narrower tiles give more, smaller work items (small frames), wider ones
 * fewer tensor-core instructions per vector; the serving loop's autotuner picks
 * it per request size.  No counterpart in the reference (its sqfnD launch shape
 * is fixed, sq.cuf:175-186). */
TRJ_API int trj_ctx_set_sq_tile_cols(trj_ctx* ctx, int cols);

/* ---- frame layout ---------------------------------------------------- */
/* Replaces the per-frame layout of select_ncdfinput (src/core/netcdf.f90:582-692)
 * and transfer_cpu_gpu (src/core/common.cuf:368-378), on the device:
 * folds each coordinate with r -= L*int(r/L) (FP32, truncation) and writes the
 * atoms species-contiguous, in input order within a species (stable).
 *   xyz_dev      n x 3 float (device)
 *   species_dev  n int32 species index 0..nsp-1 (device)
 *   packed_dev   n x 4 float out: x, y, z, species (int bits in w)
 *   counts_dev   nsp int64 out: atoms per species
 * The context keeps the per-block counting scratch, one buffer per stream; it
 * grows (one allocation) the first time a larger frame or species count is
 * seen on that stream. */
TRJ_API int trj_frame_pack(trj_ctx* ctx, const float* xyz_dev, const int32_t* species_dev, int64_t n,
                   int nsp, const float box[3], float* packed_dev, int64_t* counts_dev,
                   void* stream);
/* trj_frame_pack with the type-to-species numbering on the device: the species
 * of atom i is lut_dev[types_dev[i]] (types 0 .. nlut-1; lut entries 0..nsp-1,
 * or -1 for a type that is not selected).  A type outside the table or mapped
 * to -1 is flagged as bad data (trj_ctx_check returns TRJ_ERR_DATA): frames
 * whose atoms are all of selected types pass straight from the trajectory's
 * type column to the device, with no per-atom host work.  Other arguments and
 * results as trj_frame_pack. */
TRJ_API int trj_frame_pack_types(trj_ctx* ctx, const float* xyz_dev, const int32_t* types_dev,
                                 const int32_t* lut_dev, int nlut, int64_t n, int nsp, const float box[3],
                                 float* packed_dev, int64_t* counts_dev, void* stream);
/* trj_frame_pack for frames that carry per-atom charges (the NetCDF variable
 * "q", read as default real by src/core/netcdf.f90:404-408): the charges are
 * written in the same order as the atoms (netcdf.f90:656-658).
 *   charge_dev         n float (device)
 *   charge_packed_dev  n float out: charge of packed atom i
 * Other arguments and results as trj_frame_pack. */
TRJ_API int trj_frame_pack_charges(trj_ctx* ctx, const float* xyz_dev, const int32_t* species_dev,
                                   const float* charge_dev, int64_t n, int nsp, const float box[3],
                                   float* packed_dev, float* charge_packed_dev, int64_t* counts_dev,
                                   void* stream);

/* trj_frame_pack without any device allocation (this entry point has no
 * counterpart in the reference).  It is for callers that may not have the
 * library allocate device memory: applications whose device memory belongs to
 * another allocator (a framework's caching allocator, a pre-sized arena) and
 * frame loops that cannot take the implicit synchronisation of cudaMalloc.
 * The per-block scratch is a fixed 1 MiB device array inside the library:
 * ceil(n/1024) * nsp must be <= 87381, larger frames get TRJ_ERR_CAPACITY.
 * Every GPU that loads the library keeps that array until the process exits.
 * The first call on a device resolves the array's address on that device
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * The address is kept for the life of the process: resetting the device
 * (cudaDeviceReset) after that first call is not supported.
 * All calls share the array and overwrite what they use: calls whose work
 * overlaps on the GPU (other streams or host threads) race on it.
 * Arguments and results are those of trj_frame_pack. */
TRJ_API int trj_frame_pack_static(trj_ctx* ctx, const float* xyz_dev, const int32_t* species_dev, int64_t n,
                                  int nsp, const float box[3], float* packed_dev, int64_t* counts_dev,
                                  void* stream);

/* ---- g_ab(r) --------------------------------------------------------- */
/* Replaces RDF_init (src/modules/rdf.cuf:51-122) with the rcrdf clip of
 * select_ncdfinput (src/core/netcdf.f90:610-617): rcrdf_eff = min(rcrdf, min(box)/2),
 * side2 = rcrdf_eff^2, lsmax = nint(rcrdf_eff/deltar)+1, all in FP32.
 * n_max: largest frame the plan will accept. */
TRJ_API int trj_rdf_plan_create(trj_ctx* ctx, int nsp, float deltar, float rcrdf, const float box[3],
                        int64_t n_max, trj_rdf_plan** out);
/* Plan for two-dimensional frames (ndim = 2; rdf2_sh, rdf.cuf:617-670, and
 * s2D2_sh, rdf.cuf:555-615): the frames are packed with z = 0 (any positive
 * box[2]); the clip uses min(box[0], box[1]); distances are (x^2 + y^2) and the
 * number-fluctuation points lie in the xy plane.  Bins as trj_rdf_plan_create
 * (bin 0, r < deltar/2, is not counted, as in 3D). */
TRJ_API int trj_rdf_plan_create_2d(trj_ctx* ctx, int nsp, float deltar, float rcrdf, const float box[3],
                                   int64_t n_max, trj_rdf_plan** out);
/* Bin rule of the plan's counts: 0 = nint(r/deltar) (rdf_sh), 1 = int(r/deltar)+1
 * (rdfxy, rdf.cuf:722, the slab g(r)); bins 1..lsmax either way. */
TRJ_API int trj_rdf_plan_set_binning(trj_rdf_plan* plan, int floor_bins);
/* Failure handling of the pair kernel (the reference prints the CUDA error and
 * stops, rdf.cuf:241-242; here a device wait that runs out sets TRJ_DEV_TIMEOUT,
 * the kernel lets its copies in flight land and returns, and trj_ctx_check then
 * reports TRJ_ERR_TIMEOUT with the context still usable).  clocks: limit of a
 * warp's wait for a staged neighbour chunk, in SM clocks, 1000..2^32 (0 = the
 * default 2^32, about 2 s).  stall_test = 1 makes each warp's first wait target a
 * barrier that nothing arrives on, so that every launch of the plan runs out after
 * `clocks`: a way to exercise the timeout path without a fault.  Copies in flight
 * are always waited for with the default limit. */
TRJ_API int trj_rdf_plan_set_wait(trj_rdf_plan* plan, int64_t clocks, int stall_test);
/* Plan with nbins bins of width r_max/nbins covering [0, r_max): bin k (1-based)
 * holds r in [(k-1) dr, k dr), i.e. index floor(r/dr)+1, pairs counted for
 * rr2 < r_max^2 (FP32).  This is the binning of the freud RDF used by the
 * reference's tools/fast_grfreud_netcdf.py (bins on [0, r_max)); r_max must be
 * below half the smallest box edge. */
TRJ_API int trj_rdf_plan_create_floor(trj_ctx* ctx, int nsp, float r_max, int nbins, const float box[3],
                                      int64_t n_max, trj_rdf_plan** out);
/* lsmax, nit = nsp(nsp+1)/2, cells per axis (1 = no cell split on that axis),
 * effective cutoff, side2, device scratch bytes held by the plan. */
TRJ_API int trj_rdf_plan_info(const trj_rdf_plan* plan, int* lsmax, int* nit, int cells[3],
                      float* rcrdf_eff, float* side2, int64_t* scratch_bytes);
/* Replaces RDFcomp's device part (src/modules/rdf.cuf:184-270; kernel rdf_sh
 * 426-487): adds this frame's unordered-pair counts to hist_dev
 * (uint64 [nit][lsmax]; row = ind_ij(a,b)-1 of rdf.cuf:741-753, column = bin-1)
 * and its edge statistics to edge_dev (uint64[4], may be NULL).
 * packed_dev: output of trj_frame_pack.  box: this frame's box. */
TRJ_API int trj_rdf_accumulate(trj_rdf_plan* plan, const float* packed_dev, int64_t n, const float box[3],
                       uint64_t* hist_dev, uint64_t* edge_dev, void* stream);
/* trj_rdf_accumulate with the charge-weighted histogram of the reference's
 * ex_qc branch (rdf.cuf:225-228, 469-472, 271-274): besides the counts, every
 * counted pair adds q_a*q_b to its bin, and per frame
 *   gqq_dev[bin-1] += (sum of q_a*q_b in the bin) / avq2,  avq2 = sum(q^2)/N
 * (gqq_dev: double [lsmax]; avq2 rounded to FP32 as the reference's variable).
 * charge_packed_dev: the charges written by trj_frame_pack_charges.  Products
 * and sums are FP64 (the reference adds FP32 products with FP32 atomics).  An
 * all-zero charge set gives avq2 = 0 and non-finite gqq, as in the reference.
 * The first charged call on a plan allocates 4*n_max + 8*lsmax bytes. */
TRJ_API int trj_rdf_accumulate_charged(trj_rdf_plan* plan, const float* packed_dev, const float* charge_packed_dev,
                                       int64_t n, const float box[3], uint64_t* hist_dev, uint64_t* edge_dev,
                                       double* gqq_dev, void* stream);
/* Number fluctuations of the frame last passed to trj_rdf_accumulate on this
 * plan (s2D3_sh, src/modules/rdf.cuf:489-553, run by RDFcomp when nrandom > 0):
 * nrandom points, point b drawn with the reference's generator and seed
 * (curand XORWOW, curand_init(b + 12345, 0, 0), b = 1..nrandom; x = L_x *
 * curand_uniform, then y, z), the same points every frame; for each point N_k =
 * atoms with FP32 minimum-image distance r, r^2 < side2 and nint(r/deltar) <= k,
 * k = 0..lsmax; adds sum over points of N_k to gi_dev[k] and of N_k^2 to
 * g2i_dev[k] (uint64 [lsmax+1]; exact, where the reference sums FP32).
 * points_dev: NULL, or nrandom x 3 floats out (the sample points).
 * s2n(r_k) = g2i[k]/(Nconf nrandom) - (gi[k]/(Nconf nrandom))^2 (log.f90:532). */
TRJ_API int trj_rdf_s2n(trj_rdf_plan* plan, int nrandom, uint64_t* gi_dev, uint64_t* g2i_dev, float* points_dev,
                        void* stream);
/* Duration (ms) of the last cell-pair kernel launch; needs trj_ctx_set_timing(ctx, 1). */
TRJ_API int trj_rdf_kernel_ms(trj_rdf_plan* plan, float* ms);
TRJ_API int trj_rdf_plan_destroy(trj_rdf_plan* plan);

/* ---- S_ab(Q) --------------------------------------------------------- */
/* Replaces sq_init (src/modules/sq.cuf:150-369) given the k-set it builds:
 * nvec integer lattice vectors n (k = 2*pi*n/L per axis), each with an output
 * bin (0..nbins-1) and a weight (multiplicity; 2 for a vector standing for
 * +k and -k).  dense[v] != 0 marks vectors of a compact region that the
 * tensor-core method may evaluate through separable phase tiles; the others
 * are evaluated by the direct sum in either method.
 * species_counts: atoms per species of the frames to come (host, nsp). */
TRJ_API int trj_sq_plan_create(trj_ctx* ctx, int nsp, int64_t nvec, const int32_t* vec_host,
                       const int32_t* bin_host, const double* weight_host,
                       const uint8_t* dense_host, int nbins, const int64_t* species_counts,
                       trj_sq_plan** out);
/* Vectors evaluated by tensor tiles, tile count, padded tile work (k-slots),
 * device scratch bytes held by the plan. */
TRJ_API int trj_sq_plan_info(const trj_sq_plan* plan, int64_t* n_dense, int64_t* n_tiles,
                     int64_t* tile_slots, int64_t* scratch_bytes);
/* Tensor-core tuning: atoms accumulated by the tensor cores in one FP32 run before
 * the run is added (round-to-nearest) into the running sum, rounded down to a
 * multiple of 32 (>= 32).  The tensor-core accumulation error grows linearly with
 * the run length, so longer runs trade accuracy for fewer drains; the default,
 * 256 atoms, keeps the per-shell error of an N = 1e6 frame below 1e-5. */
TRJ_API int trj_sq_plan_set_flush(trj_sq_plan* plan, int atoms);
/* Tensor-core tuning: evaluate pairs of tiles that share their nz range as one
 * M = 256 contraction on a cluster of two CTAs (tcgen05 cta_group::2, each SM
 * holding half of the shared operand and its running sum in shared memory) when
 * enable != 0, or each tile on one CTA when 0 (the default, faster on the
 * N = 1e6 benchmark frame).  Both give the same sums.  The pair form is used
 * only where the device keeps clusters of two resident. */
TRJ_API int trj_sq_plan_set_pairs(trj_sq_plan* plan, int enable);
/* Replaces SQcalc (src/modules/sq.cuf:58-126; kernels sqfnD 523-591, sqfact
 * 372-454): adds, for every bin and species pair (a<=b, row ind_ij(a,b)-1),
 * sum over the bin's vectors of weight * Re(rho_a(k) conj(rho_b(k))) to
 * out_dev (double [nbins][nit]), rho_a(k) = sum_{j in a} exp(i k.r_j).
 * method: TRJ_SQ_PLAIN_FP32 or TRJ_SQ_SPLIT_BF16X3. */
TRJ_API int trj_sq_accumulate(trj_sq_plan* plan, const float* packed_dev, int64_t n, const float box[3],
                      int method, double* out_dev, void* stream);
/* Plan for frames with charges (the reference's ex_qc S(Q), sq.cuf:67, 569-588,
 * 143-145): arguments as trj_sq_plan_create (nsp <= 15), and the plan adds a
 * species nsp, the charge density rho_q(k) = sum_j q_j exp(i k.r_j) over every
 * atom.  Its accumulate output has nit = (nsp+1)(nsp+2)/2 rows: the species
 * pairs, the cross rows (a, nsp) and, in the last row (nsp, nsp), the sums of
 * w |rho_q(k)|^2, the reference's sqfq_d before its division by
 * avq2 = sum(q^2)/N.  trj_sq_rho gives nsp+1 densities. */
TRJ_API int trj_sq_plan_create_charged(trj_ctx* ctx, int nsp, int64_t nvec, const int32_t* vec_host,
                                       const int32_t* bin_host, const double* weight_host,
                                       const uint8_t* dense_host, int nbins, const int64_t* species_counts,
                                       trj_sq_plan** out);
/* trj_sq_accumulate for a charged plan; charge_packed_dev as written by
 * trj_frame_pack_charges.  A charged plan accepts only this call. */
TRJ_API int trj_sq_accumulate_charged(trj_sq_plan* plan, const float* packed_dev, const float* charge_packed_dev,
                                      int64_t n, const float box[3], int method, double* out_dev, void* stream);
/* Planar frames in tile form (mul > 0): every atom's third phase coordinate is
 * taken as mul * (its second) mod 1, exactly in 32-bit fixed point, instead of
 * its z.  A plan whose vectors are (nx, ny mod mul, ny div mul) then evaluates
 * the in-plane vectors (nx, ny) of a z = 0 frame, and 16 x 8 x nz tensor tiles
 * fill with them (ndim = 2 S(Q) on the tensor path).  0 turns it off. */
TRJ_API int trj_sq_plan_set_z_from_y(trj_sq_plan* plan, int mul);
/* Direct sums over caller-defined atom groups, for the plan's vectors:
 * rho_g(k) = sum over atoms j in group g of exp(i k.r_j), FP64 [ngroups][nvec][2]
 * in the caller's vector order.  packed_dev holds n atoms (x, y, z; w unused)
 * with the groups contiguous: group g = atoms group_off_host[g] ..
 * group_off_host[g+1]-1 (host array of ngroups+1 offsets, 0 .. n).  Groups may
 * change from call to call; this is how the slab S(Q) (sqf3xy/sqf2xy,
 * sq.cuf:594-771) forms the density of every species in every z slice.  FP32
 * terms of exactly reduced phases, FP64 sums (the direct-sum path). */
TRJ_API int trj_sq_rho_groups(trj_sq_plan* plan, const float* packed_dev, int64_t n, const float box[3],
                              int ngroups, const int64_t* group_off_host, double* rho_out, void* stream);
/* rho_a(k) of the last accumulate, FP64, [nsp][nvec][2] in the caller's vector order. */
TRJ_API int trj_sq_rho(trj_sq_plan* plan, double* rho_dev, void* stream);
/* Duration (ms) of the last main S(Q) kernel launch (tcgen05 contraction for
 * TRJ_SQ_SPLIT_BF16X3, direct sum for TRJ_SQ_PLAIN_FP32); needs timing enabled. */
TRJ_API int trj_sq_kernel_ms(trj_sq_plan* plan, float* ms);
TRJ_API int trj_sq_plan_destroy(trj_sq_plan* plan);

/* ---- F(Q,t), Fs(Q,t), mean-squared displacement ------------------------ */
/* Replaces the device part of dyn_init/rtcorr (src/modules/dynamics.cuf:88-135,
 * 157-276; kernels FqtnD 421-507 and rtcal 510-547).  nbuffer time origins, each
 * with ndyn lag rows; nvec integer lattice vectors n (k = 2*pi*n/L per axis) with
 * their output bins 0..nbins-1 (the qw shells of sq.cuf:239-297); bsc: the
 * coherent weight per species; n: atoms per frame (same order in every frame, as
 * trj_frame_pack writes them).  Device memory: about 48*nbuffer*n bytes plus the
 * accumulators (3 x nbuffer*ndyn*nbins doubles). */
TRJ_API int trj_dyn_plan_create(trj_ctx* ctx, int nsp, int64_t n, int nbuffer, int ndyn, int64_t nvec,
                                const int32_t* vec_host, const int32_t* bin_host, int nbins,
                                const float* bsc_host, trj_dyn_plan** out);
TRJ_API int trj_dyn_plan_info(const trj_dyn_plan* plan, int64_t* scratch_bytes);
/* One frame: for every buffer b with lag_host[b] >= 0 (0-based lag row,
 * < ndyn; -1 = buffer not started or finished) adds to its rows
 *   F_b(bin, lag)  += sum over the bin's k of Re(rho(k,t0) conj(rho(k,t))),
 *                     rho(k,t) = sum_j bsc[species_j] exp(i k.r_j(t))
 *   Fs_b(bin, lag) += sum over the bin's k of sum_j cos(k.(r_j(t) - r_j(t0)))
 *   C_b(lag)       += sum_j |rt_j(t) - r_j(t0)|^2 / n   (rt unwrapped per buffer)
 * origin_host[b] = 1 makes this frame buffer b's origin t0 (its lag must be 0).
 * packed_dev: output of trj_frame_pack for this frame. */
TRJ_API int trj_dyn_accumulate(trj_dyn_plan* plan, const float* packed_dev, int64_t n, const float box[3],
                               const int32_t* lag_host, const uint8_t* origin_host, void* stream);
/* Adds the rows of every buffer with done_host[b] = 1 to the totals and clears
 * them (rtcorr, dynamics.cuf:239-269): fkt_dev, fskt_dev double [ndyn][nbins],
 * r2t_dev double [ndyn]. */
TRJ_API int trj_dyn_flush(trj_dyn_plan* plan, const uint8_t* done_host, double* fkt_dev, double* fskt_dev,
                          double* r2t_dev, void* stream);
/* Duration (ms) of the last self-term kernel launch; needs timing enabled. */
TRJ_API int trj_dyn_kernel_ms(trj_dyn_plan* plan, float* ms);
TRJ_API int trj_dyn_plan_destroy(trj_dyn_plan* plan);

/* ---- Fused launches over several small requests ------------------------- */
/* The reference runs one frame of one system per step of its main loop
 * (src/main/trj_analysis.f90:208-217: transfer_cpu_gpu, then RDFcomp's rdf_sh
 * launch rdf.cuf:240 and SQcalc's sqfnD launch sq.cuf:89).  A batch runs one
 * frame of each of up to max_items requests per turn through one fixed launch
 * sequence: a copy of the turn's descriptor table, frame layout (fold, species
 * order, fixed-point phases; select_ncdfinput), an all-pairs histogram with
 * rdf_sh's arithmetic (rdf.cuf:449-475) and the FP32 direct sum with FP64 shell
 * sums (the plain method of trj_sq_accumulate), every kernel over the work of
 * all the turn's frames.  The sequence does not depend on what the table holds,
 * so a CUDA graph captured once per staging buffer replays every later turn.
 * Two staging buffers (0, 1) let the host fill one turn while the device runs
 * the other; the caller orders each buffer's reuse after its previous launch
 * (an event), since the table and the staged atoms are read when the launch
 * executes.  Counts are those of trj_rdf_accumulate and S(Q) sums those of
 * trj_sq_accumulate(TRJ_SQ_PLAIN_FP32) for the same plans, bit for bit.
 * max_atoms: staged atoms per turn; hist_words: the largest nit*lsmax of a
 * pair plan the batch takes (shared memory: 8 bytes per word + 4 KB). */
TRJ_API int trj_batch_create(trj_ctx* ctx, int max_items, int64_t max_atoms, int hist_words, trj_batch** out);
/* Host staging of buffer buf: xyz[3 * max_atoms] float and species[max_atoms]
 * int32 (0-based species ids), pinned and mapped into the device's address
 * space: the layout kernel reads them directly. */
TRJ_API int trj_batch_staging(trj_batch* batch, int buf, float** xyz_host, int32_t** species_host);
/* Starts a new turn in buffer buf (no items). */
TRJ_API int trj_batch_begin(trj_batch* batch, int buf);
/* Adds one frame of one request: atoms [atom_off, atom_off + n) of the
 * staging, items in increasing atom order.  rdf: the request's pair plan (its
 * cutoff, clipped per frame as trj_rdf_accumulate does, bins and species; its
 * cell arrays are not used, so it may be created with n_max 0) or NULL; sq: its
 * S(Q) plan (uncharged; species counts summing to n; its partial-sum scratch is
 * used) or NULL.  Accumulates into hist_dev ([nit][lsmax] uint64), edge_dev
 * (TRJ_EDGE_* counters, may be NULL) and sq_out_dev ([nbins][nit] double) as
 * the single-request calls do.  TRJ_ERR_UNSUPPORTED: a plan that runs only
 * unfused (charged, two-dimensional, nit*lsmax > hist_words, > 16 species). */
TRJ_API int trj_batch_add(trj_batch* batch, int buf, trj_rdf_plan* rdf, trj_sq_plan* sq, int64_t atom_off,
                          int64_t n, const float box[3], uint64_t* hist_dev, uint64_t* edge_dev,
                          double* sq_out_dev);
/* Enqueues the turn of buffer buf on stream: one table copy and five kernels. */
TRJ_API int trj_batch_launch(trj_batch* batch, int buf, void* stream);
/* Items and work units (layout, pair tiles, direct-sum blocks, shell bins) of
 * buffer buf's turn; device memory the batch holds. */
TRJ_API int trj_batch_info(const trj_batch* batch, int buf, int* nitems, int64_t units[4], int64_t* device_bytes);
/* Duration (ms) of the last launched turn's kernels; needs timing enabled. */
TRJ_API int trj_batch_kernel_ms(trj_batch* batch, float* ms);
/* Waits for the device, then frees the staging and device memory. */
TRJ_API int trj_batch_destroy(trj_batch* batch);

#ifdef __cplusplus
}
#endif
#endif /* TRJ_SM100_H */
