/*
 * oracle.c -- CPU restatement of the reference's g_ab(r) and S_ab(Q) arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product path links, loads or calls
 * this file; only tests/, the smoke check and bench.py's CPU-baseline leg do,
 * and only as the checker (or as the timed CPU baseline).
 *
 * Compiled with -ffp-contract=off so that every FP32 expression rounds once per
 * operation in the order written (no fused multiply-add), as the reference's
 * Fortran states it.
 *
 * Reference functions restated here (file:line within the reference project):
 *   pair arithmetic      src/modules/rdf.cuf:451-475   (rdf_sh inner loop)
 *   pair index           src/modules/rdf.cuf:741-753   (ind_ij)
 *   histogram layout     src/modules/rdf.cuf:51-66     (lsmax = nint(rcrdf/deltar)+1)
 *   S(Q) direct sum      src/modules/sq.cuf:523-591    (sqfnD; FP32 phase, FP64 sums)
 *                        src/modules/sq.cuf:372-454    (sqfact; axis vectors)
 *   charge products      src/modules/rdf.cuf:469-472   (gqq_d(ind) += qci*qcj, ex_qc)
 *   charge density       src/modules/sq.cuf:569-573    (sumqcx += qci*cfk, ex_qc)
 *
 * The exact S(Q) oracle is FP64 throughout: phases from the fractional
 * coordinate s = x/L in FP64, n.s reduced mod 1 in FP64, sin/cos in FP64.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------ */
/* g(r): reference pair arithmetic                                     */
/* ------------------------------------------------------------------ */

typedef struct {
    float L[3];
    float side2;
    float deltar;
    int lsmax;
    int nsp;
    int floor_bins;  /* 0: nint(r/deltar) as rdf_sh; 1: floor(r/deltar)+1 (bins [k dr, (k+1) dr)) */
} orc_rdf_params;

static int g_floor_bins = 0;  /* binning of the next orc_rdf_* call (set by orc_set_binning) */

ORC_EXPORT void orc_set_binning(int floor_bins) { g_floor_bins = floor_bins; }

/* ind_ij (rdf.cuf:741-753), 0-based species a,b -> 0-based pair row. */
static inline int pair_row(int a, int b, int nsp) {
    if (a > b) { int t = a; a = b; b = t; }
    return a * (nsp - 1) - a * (a - 1) / 2 + b;
}

/* xd = xd - sidel*nint(xd/sidel)  (rdf.cuf:457-459); NINT rounds half away from zero. */
static inline float min_image(float d, float L) {
    float q = d / L;
    float n = roundf(q);
    float s = L * n;
    return d - s;
}

/* Outcome of one pair: bin 1..lsmax, or 0 when not counted (rdf.cuf:461-467). */
static inline int pair_outcome(float rr2, const orc_rdf_params* p) {
    if (!(rr2 < p->side2)) return 0;
    float rr = sqrtf(rr2);
    float q = rr / p->deltar;
    int ind = p->floor_bins ? (int)floorf(q) + 1 : (int)roundf(q);
    if (ind <= p->lsmax && ind > 0) return ind;
    return 0;
}

typedef struct {
    uint64_t edge_ulp;   /* outcome changes when rr2 moves by one FP32 ulp */
    uint64_t edge_fma;   /* outcome changes under the FMA-contracted rr2    */
    uint64_t counted;    /* pairs counted into the histogram               */
} orc_edge_stats;

/* One unordered pair: accumulate its count and edge statistics; returns its bin (0: not counted). */
static inline int do_pair(const float* pi, int si, const float* pj, int sj,
                          const orc_rdf_params* p, uint64_t* hist, orc_edge_stats* e) {
    float xd = pj[0] - pi[0];
    float yd = pj[1] - pi[1];
    float zd = pj[2] - pi[2];
    xd = min_image(xd, p->L[0]);
    yd = min_image(yd, p->L[1]);
    zd = min_image(zd, p->L[2]);
    float x2 = xd * xd, y2 = yd * yd, z2 = zd * zd;
    float rr2 = (x2 + y2) + z2;
    /* Anything at or beyond 1.001*side2 cannot reach the cutoff by an ulp or by FMA. */
    if (!(rr2 < p->side2 * 1.001f)) return 0;
    int o = pair_outcome(rr2, p);
    if (o) {
        hist[(size_t)pair_row(si, sj, p->nsp) * p->lsmax + (o - 1)] += 1;
        e->counted += 1;
    }
    int olo = pair_outcome(nextafterf(rr2, -INFINITY), p);
    int ohi = pair_outcome(nextafterf(rr2, INFINITY), p);
    if (olo != o || ohi != o) e->edge_ulp += 1;
    float rr2f = fmaf(zd, zd, fmaf(yd, yd, x2));
    if (pair_outcome(rr2f, p) != o) e->edge_fma += 1;
    return o;
}

/* Charge product of a counted pair, added in FP64 (the product of two FP32 values is exact). */
static inline void add_charge(int o, const float* q, int64_t i, int64_t j, double* gq) {
    if (o && q) gq[o - 1] += (double)q[i] * (double)q[j];
}

/*
 * All-pairs g(r) over one frame (the reference's O(N^2) algorithm).
 * pos: N x 3 FP32 (already folded, species-contiguous or not: order is irrelevant).
 * sp:  N species indices (0-based).
 * hist: nit x lsmax uint64, accumulated (+=).
 */
static void rdf_allpairs_impl(const float* pos, const int32_t* sp, const float* q, int64_t n,
                              const float box[3], float side2, float deltar, int lsmax, int nsp,
                              uint64_t* hist, uint64_t* edge3, double* gqq) {
    orc_rdf_params p = {{box[0], box[1], box[2]}, side2, deltar, lsmax, nsp, g_floor_bins};
    int nit = nsp * (nsp + 1) / 2;
    int nthr = 1;
#ifdef _OPENMP
    nthr = omp_get_max_threads();
#endif
    size_t hsz = (size_t)nit * lsmax;
    uint64_t* priv = (uint64_t*)calloc((size_t)nthr * hsz, sizeof(uint64_t));
    double* qpriv = (double*)calloc((size_t)nthr * lsmax, sizeof(double));
    orc_edge_stats* es = (orc_edge_stats*)calloc((size_t)nthr, sizeof(orc_edge_stats));
#pragma omp parallel
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        uint64_t* h = priv + (size_t)t * hsz;
        double* gq = qpriv + (size_t)t * lsmax;
#pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < n; ++i)
            for (int64_t j = i + 1; j < n; ++j)
                add_charge(do_pair(pos + 3 * i, sp[i], pos + 3 * j, sp[j], &p, h, &es[t]), q, i, j, gq);
    }
    for (int t = 0; t < nthr; ++t) {
        for (size_t k = 0; k < hsz; ++k) hist[k] += priv[(size_t)t * hsz + k];
        if (gqq)
            for (int k = 0; k < lsmax; ++k) gqq[k] += qpriv[(size_t)t * lsmax + k];
        edge3[0] += es[t].edge_ulp;
        edge3[1] += es[t].edge_fma;
        edge3[2] += es[t].counted;
    }
    free(priv);
    free(qpriv);
    free(es);
}

ORC_EXPORT void orc_rdf_allpairs(const float* pos, const int32_t* sp, int64_t n,
                                 const float box[3], float side2, float deltar,
                                 int lsmax, int nsp, uint64_t* hist, uint64_t* edge3) {
    rdf_allpairs_impl(pos, sp, NULL, n, box, side2, deltar, lsmax, nsp, hist, edge3, NULL);
}

/*
 * Linked-cell g(r) with identical per-pair arithmetic.  Cells are built from
 * the wrapped coordinate; a pair is tested once, from its lower original index,
 * over the 27-cell neighbourhood.  Requires >= 3 cells per axis (else falls
 * back to all pairs).  Cell edge >= rcut*(1+2^-10) so that no pair whose FP32
 * rr2 is below side2 is outside the neighbourhood.
 */
/* Same, restricted to home atoms i in [i0, i1) (pairs (i, j>i)); used to time a bounded
 * sample of a large frame for the CPU baseline.  i0=0, i1=n is the whole frame. */
static void rdf_cells_impl(const float* pos, const int32_t* sp, const float* q, int64_t n,
                           const float box[3], float side2, float deltar, int lsmax, int nsp,
                           uint64_t* hist, uint64_t* edge3, double* gqq, int64_t i0, int64_t i1);

ORC_EXPORT void orc_rdf_cells(const float* pos, const int32_t* sp, int64_t n,
                              const float box[3], float side2, float deltar,
                              int lsmax, int nsp, uint64_t* hist, uint64_t* edge3) {
    rdf_cells_impl(pos, sp, NULL, n, box, side2, deltar, lsmax, nsp, hist, edge3, NULL, 0, n);
}

ORC_EXPORT void orc_rdf_cells_range(const float* pos, const int32_t* sp, int64_t n,
                                    const float box[3], float side2, float deltar,
                                    int lsmax, int nsp, uint64_t* hist, uint64_t* edge3,
                                    int64_t i0, int64_t i1) {
    rdf_cells_impl(pos, sp, NULL, n, box, side2, deltar, lsmax, nsp, hist, edge3, NULL, i0, i1);
}

/* Counts plus gqq[bin-1] += sum over counted pairs of q_i*q_j (FP64, not divided by avq2);
 * cells != 0 takes the linked-cell sweep. */
ORC_EXPORT void orc_rdf_charged(const float* pos, const int32_t* sp, const float* q, int64_t n,
                                const float box[3], float side2, float deltar, int lsmax, int nsp,
                                uint64_t* hist, uint64_t* edge3, double* gqq, int cells) {
    if (cells) rdf_cells_impl(pos, sp, q, n, box, side2, deltar, lsmax, nsp, hist, edge3, gqq, 0, n);
    else rdf_allpairs_impl(pos, sp, q, n, box, side2, deltar, lsmax, nsp, hist, edge3, gqq);
}

static void rdf_cells_impl(const float* pos, const int32_t* sp, const float* q, int64_t n,
                           const float box[3], float side2, float deltar, int lsmax, int nsp,
                           uint64_t* hist, uint64_t* edge3, double* gqq, int64_t i0, int64_t i1) {
    double rc = sqrt((double)side2) * (1.0 + 1.0 / 1024.0);
    int nc[3];
    for (int d = 0; d < 3; ++d) {
        nc[d] = (int)floor((double)box[d] / rc);
        if (nc[d] < 3) { rdf_allpairs_impl(pos, sp, q, n, box, side2, deltar, lsmax, nsp, hist, edge3, gqq); return; }
    }
    int64_t ncell = (int64_t)nc[0] * nc[1] * nc[2];
    int64_t* head = (int64_t*)malloc(sizeof(int64_t) * ncell);
    int64_t* next = (int64_t*)malloc(sizeof(int64_t) * n);
    int32_t* cellof = (int32_t*)malloc(sizeof(int32_t) * n * 3);
    for (int64_t c = 0; c < ncell; ++c) head[c] = -1;
    for (int64_t i = n - 1; i >= 0; --i) {
        int cc[3];
        for (int d = 0; d < 3; ++d) {
            double L = box[d];
            double w = (double)pos[3 * i + d];
            w = w - L * floor(w / L);
            int k = (int)floor(w / L * nc[d]);
            if (k < 0) k = 0;
            if (k >= nc[d]) k = nc[d] - 1;
            cc[d] = k;
            cellof[3 * i + d] = k;
        }
        int64_t c = ((int64_t)cc[0] * nc[1] + cc[1]) * nc[2] + cc[2];
        next[i] = head[c];
        head[c] = i;
    }
    orc_rdf_params p = {{box[0], box[1], box[2]}, side2, deltar, lsmax, nsp, g_floor_bins};
    int nit = nsp * (nsp + 1) / 2;
    int nthr = 1;
#ifdef _OPENMP
    nthr = omp_get_max_threads();
#endif
    size_t hsz = (size_t)nit * lsmax;
    uint64_t* priv = (uint64_t*)calloc((size_t)nthr * hsz, sizeof(uint64_t));
    double* qpriv = (double*)calloc((size_t)nthr * lsmax, sizeof(double));
    orc_edge_stats* es = (orc_edge_stats*)calloc((size_t)nthr, sizeof(orc_edge_stats));
#pragma omp parallel
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        uint64_t* h = priv + (size_t)t * hsz;
        double* gq = qpriv + (size_t)t * lsmax;
#pragma omp for schedule(dynamic, 256)
        for (int64_t i = i0; i < i1; ++i) {
            for (int dx = -1; dx <= 1; ++dx)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dz = -1; dz <= 1; ++dz) {
                        int cx = (cellof[3 * i] + dx + nc[0]) % nc[0];
                        int cy = (cellof[3 * i + 1] + dy + nc[1]) % nc[1];
                        int cz = (cellof[3 * i + 2] + dz + nc[2]) % nc[2];
                        int64_t c = ((int64_t)cx * nc[1] + cy) * nc[2] + cz;
                        for (int64_t j = head[c]; j >= 0; j = next[j])
                            if (j > i)
                                add_charge(do_pair(pos + 3 * i, sp[i], pos + 3 * j, sp[j], &p, h, &es[t]), q, i, j,
                                           gq);
                    }
        }
    }
    for (int t = 0; t < nthr; ++t) {
        for (size_t k = 0; k < hsz; ++k) hist[k] += priv[(size_t)t * hsz + k];
        if (gqq)
            for (int k = 0; k < lsmax; ++k) gqq[k] += qpriv[(size_t)t * lsmax + k];
        edge3[0] += es[t].edge_ulp;
        edge3[1] += es[t].edge_fma;
        edge3[2] += es[t].counted;
    }
    free(priv);
    free(qpriv);
    free(es);
    free(head);
    free(next);
    free(cellof);
}

/* ------------------------------------------------------------------ */
/* S(Q): exact FP64 rho_a(k)                                           */
/* ------------------------------------------------------------------ */

/*
 * rho[a][v] = sum_{j in species a} exp(i 2 pi n_v . s_j),  s_j = x_j / L (FP64).
 * pos: N x 3 FP32 species-contiguous; sp_off: nsp+1 offsets; vec: nvec x 3 ints.
 * rho: nsp x nvec x 2 doubles (re, im), overwritten.
 *
 * Separable evaluation: per block of atoms, e^{i 2 pi n s} for every needed n on
 * each axis is a direct FP64 cos/sin of the reduced fraction n s - nint(n s),
 * stored per axis value as contiguous runs over the block's atoms.  Vectors are
 * grouped by (nx, ny): the FP64 product X Y of a group is formed once per atom
 * and multiplied by Z for each nz of the group.  Sums are FP64 (four partial
 * sums per vector inside a block, then per block and per thread).
 */
static void rho_fp64_impl(const float* pos, const float* w, int64_t n, const int64_t* sp_off, int nsp,
                          const float box[3], int64_t nvec, const int32_t* vec, double* rho);

ORC_EXPORT void orc_rho_fp64(const float* pos, int64_t n, const int64_t* sp_off, int nsp,
                             const float box[3], int64_t nvec, const int32_t* vec, double* rho) {
    rho_fp64_impl(pos, NULL, n, sp_off, nsp, box, nvec, vec, rho);
}

/* Weighted density sum_{j in a} w_j exp(i 2 pi n_v . s_j); with every atom in one range and
 * w = charges this is the charge density rho_q(k) of the reference's ex_qc S(Q). */
ORC_EXPORT void orc_rho_fp64_w(const float* pos, const float* w, int64_t n, const int64_t* sp_off, int nsp,
                               const float box[3], int64_t nvec, const int32_t* vec, double* rho) {
    rho_fp64_impl(pos, w, n, sp_off, nsp, box, nvec, vec, rho);
}

#define ORC_BLK 256                                   /* atoms per block */
typedef double orc_v4 __attribute__((vector_size(32)));  /* four doubles (plain SIMD pairs on SSE2) */

static const int32_t* g_sort_vec;
static int cmp_xy(const void* pa, const void* pb) {
    const int64_t a = *(const int64_t*)pa, b = *(const int64_t*)pb;
    const int32_t* va = g_sort_vec + 3 * a;
    const int32_t* vb = g_sort_vec + 3 * b;
    if (va[0] != vb[0]) return va[0] < vb[0] ? -1 : 1;
    if (va[1] != vb[1]) return va[1] < vb[1] ? -1 : 1;
    return a < b ? -1 : (a > b);
}

static void rho_fp64_impl(const float* pos, const float* w, int64_t n, const int64_t* sp_off, int nsp,
                          const float box[3], int64_t nvec, const int32_t* vec, double* rho) {
    (void)n;
    memset(rho, 0, sizeof(double) * 2 * (size_t)nsp * nvec);
    if (nvec == 0) return;
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int64_t v = 0; v < nvec; ++v)
        for (int d = 0; d < 3; ++d) {
            if (vec[3 * v + d] < lo[d]) lo[d] = vec[3 * v + d];
            if (vec[3 * v + d] > hi[d]) hi[d] = vec[3 * v + d];
        }
    int span[3];
    for (int d = 0; d < 3; ++d) span[d] = hi[d] - lo[d] + 1;
    const int tsz = span[0] + span[1] + span[2];
    /* vectors sorted by (nx, ny); groups of equal (nx, ny) */
    int64_t* ord = (int64_t*)malloc(sizeof(int64_t) * (size_t)nvec);
    for (int64_t v = 0; v < nvec; ++v) ord[v] = v;
    g_sort_vec = vec;
    qsort(ord, (size_t)nvec, sizeof(int64_t), cmp_xy);
    int64_t* gstart = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nvec + 1));
    int64_t ng = 0;
    for (int64_t k = 0; k < nvec; ++k) {
        const int32_t* a = vec + 3 * ord[k];
        if (k == 0 || a[0] != vec[3 * ord[k - 1]] || a[1] != vec[3 * ord[k - 1] + 1]) gstart[ng++] = k;
    }
    gstart[ng] = nvec;
    int nthr = 1;
#ifdef _OPENMP
    nthr = omp_get_max_threads();
#endif
    for (int a = 0; a < nsp; ++a) {
        const int64_t j0 = sp_off[a], j1 = sp_off[a + 1];
        const int64_t nblk = (j1 - j0 + ORC_BLK - 1) / ORC_BLK;
        double* acc = (double*)calloc((size_t)nthr * nvec * 2, sizeof(double));
#pragma omp parallel
        {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            double* my = acc + (size_t)t * nvec * 2;
            /* table [axis value][re/im][ORC_BLK], zero past the block's atoms */
            double* tab = (double*)aligned_alloc(64, sizeof(double) * 2 * (size_t)tsz * ORC_BLK);
            double* ar = (double*)aligned_alloc(64, sizeof(double) * ORC_BLK);
            double* ai = (double*)aligned_alloc(64, sizeof(double) * ORC_BLK);
#pragma omp for schedule(dynamic, 1)
            for (int64_t b = 0; b < nblk; ++b) {
                const int64_t jb = j0 + b * ORC_BLK, je = jb + ORC_BLK < j1 ? jb + ORC_BLK : j1;
                const int cnt = (int)(je - jb);
                int base = 0;
                for (int d = 0; d < 3; ++d) {
                    for (int m = 0; m < span[d]; ++m) {
                        double* re = tab + (size_t)(base + m) * 2 * ORC_BLK;
                        double* im = re + ORC_BLK;
                        for (int q = 0; q < ORC_BLK; ++q) {
                            if (q < cnt) {
                                const double s = (double)pos[3 * (jb + q) + d] / (double)box[d];
                                double t2 = (double)(m + lo[d]) * s;
                                t2 -= nearbyint(t2);
                                const double ang = 2.0 * M_PI * t2;
                                /* the weight rides on the z factor */
                                const double wq = (d == 2 && w) ? (double)w[jb + q] : 1.0;
                                re[q] = wq * cos(ang);
                                im[q] = wq * sin(ang);
                            } else {
                                re[q] = 0.0;
                                im[q] = 0.0;
                            }
                        }
                    }
                    base += span[d];
                }
                for (int64_t g = 0; g < ng; ++g) {
                    const int32_t* v0 = vec + 3 * ord[gstart[g]];
                    const double* xr = tab + (size_t)(v0[0] - lo[0]) * 2 * ORC_BLK;
                    const double* xi = xr + ORC_BLK;
                    const double* yr = tab + (size_t)(span[0] + v0[1] - lo[1]) * 2 * ORC_BLK;
                    const double* yi = yr + ORC_BLK;
                    for (int q = 0; q < ORC_BLK; ++q) {
                        ar[q] = xr[q] * yr[q] - xi[q] * yi[q];
                        ai[q] = xr[q] * yi[q] + xi[q] * yr[q];
                    }
                    for (int64_t k = gstart[g]; k < gstart[g + 1]; ++k) {
                        const int64_t v = ord[k];
                        const double* zr = tab + (size_t)(span[0] + span[1] + vec[3 * v + 2] - lo[2]) * 2 * ORC_BLK;
                        const double* zi = zr + ORC_BLK;
                        orc_v4 sr = {0, 0, 0, 0}, si = {0, 0, 0, 0};
                        for (int q = 0; q < ORC_BLK; q += 4) {
                            orc_v4 a_r, a_i, z_r, z_i;
                            memcpy(&a_r, ar + q, 32);
                            memcpy(&a_i, ai + q, 32);
                            memcpy(&z_r, zr + q, 32);
                            memcpy(&z_i, zi + q, 32);
                            sr += a_r * z_r - a_i * z_i;
                            si += a_r * z_i + a_i * z_r;
                        }
                        my[2 * v] += (sr[0] + sr[1]) + (sr[2] + sr[3]);
                        my[2 * v + 1] += (si[0] + si[1]) + (si[2] + si[3]);
                    }
                }
            }
            free(tab);
            free(ar);
            free(ai);
        }
        for (int t = 0; t < nthr; ++t)
            for (int64_t v = 0; v < nvec; ++v) {
                rho[((size_t)a * nvec + v) * 2] += acc[((size_t)t * nvec + v) * 2];
                rho[((size_t)a * nvec + v) * 2 + 1] += acc[((size_t)t * nvec + v) * 2 + 1];
            }
        free(acc);
    }
    free(ord);
    free(gstart);
}

/*
 * The reference's own S(Q) arithmetic on the CPU (sqfnD, sq.cuf:537-581):
 * kf = n*fk in FP32, phase = (y*kf2 + x*kf1) + z*kf3 in FP32, cos/sin of that
 * FP32 phase (libm sinf/cosf here, the GPU intrinsics __cosf/__sinf there),
 * FP64 sums per species.  Used as the timed CPU baseline, not as truth.
 * rho: nsp x nvec x 2 doubles, overwritten.
 */
ORC_EXPORT void orc_rho_ref32(const float* pos, int64_t n, const int64_t* sp_off, int nsp,
                              const float box[3], int64_t nvec, const int32_t* vec, double* rho) {
    const float twopi = 2.0f * 3.14159274f;
    float fk[3] = {twopi / box[0], twopi / box[1], twopi / box[2]};
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t v = 0; v < nvec; ++v) {
        float kf1 = (float)vec[3 * v] * fk[0];
        float kf2 = (float)vec[3 * v + 1] * fk[1];
        float kf3 = (float)vec[3 * v + 2] * fk[2];
        for (int a = 0; a < nsp; ++a) {
            double sc = 0.0, ss = 0.0;
            for (int64_t j = sp_off[a]; j < sp_off[a + 1]; ++j) {
                const float* r = pos + 3 * j;
                float ph = r[1] * kf2 + r[0] * kf1;
                ph = ph + r[2] * kf3;
                sc += (double)cosf(ph);
                ss += (double)sinf(ph);
            }
            rho[((size_t)a * nvec + v) * 2] = sc;
            rho[((size_t)a * nvec + v) * 2 + 1] = ss;
        }
    }
}

ORC_EXPORT int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
