/*
 * compact_oracle.c -- CPU restatement of the reference's compact-hashing fixed-radius
 * neighbour search.  TEST INFRASTRUCTURE ONLY: it is the checker that the CUDA path is
 * compared against (tests/, __graft_entry__.smoke, bench.py's cpu_baseline leg); no product
 * code loads it.
 *
 * What it restates (reference paths relative to src/torchCompactRadius/):
 *   - periodic wrap            util.py:375-387 (radiusSearch, once per cloud) and
 *                              compactHashing/cppSearch.py:221 (reference cloud, a second time);
 *                              torch.remainder = fmod, then +b when the signs differ.
 *   - grid support hMax        compactHashing/cellTable.py:40-81 (computeGridSupport)
 *   - cell size hCell          util.py:28-79 (compute_h), float32 tensor arithmetic
 *   - cell counts / indices    compactHashing/cellTable.py:27-31 and util.py:176-193
 *   - cell table + hash table  compactHashing/hashTable.py:159-234 (buildCompactHashMap_compat)
 *   - hash                     cppSrc/hashing.h:20-34 (uint32 wrap-around, primes 73856093,
 *                              19349663, 83492791; 1-D is c mod L)
 *   - stencil order            cppSrc/neighborhoodDynamic_cpu.cpp:153-177 (last coord fastest)
 *   - lookup                   cppSrc/neighborhood.h:13-94 (linear index match inside the
 *                              bucket of the stencil cell's hash; pymod wrap on periodic dims)
 *   - distance / modes         cppSrc/common.h:95-129 and cppSrc/neighborhoodDynamic.h:37-115:
 *                              per dim diff in double (moduloOp for periodic dims, float
 *                              subtraction widened otherwise), sum = (float)((double)sum +
 *                              diff*diff), dist = sqrtf(sum), strict '<' against
 *                              gather h_i / scatter h_j / symmetric (h_i+h_j)/2.f /
 *                              superSymmetric max(h_i,h_j).
 *   - output                   rows in query order, j = sortIndex[j_sorted]
 *                              (cppSearch.py:74-97) and CSR counts (util.py:335-358).
 *
 * Sorting here is stable (ties broken by index), so the cell table is deterministic.  The
 * reference's torch.argsort is not stable, which only changes the order of points inside a
 * cell and of cells inside a hash bucket, never the pair set -- except when two different
 * occupied cells share one int32 linear index (points outside a non-periodic domain), where
 * the reference's own result depends on its sort order.
 *
 * Build: see oracle/Makefile (-O2 -ffp-contract=off, no fast-math; OpenMP optional).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { OR_GATHER = 0, OR_SCATTER = 1, OR_SYMMETRIC = 2, OR_SUPERSYMMETRIC = 3 };

/* torch.remainder for float32 (ATen BinaryOpsKernel: fmod, then add b when signs differ). */
static float torch_remainder_f(float a, float b) {
    float m = fmodf(a, b);
    if (m != 0.0f && ((b < 0.0f) != (m < 0.0f))) m += b;
    return m;
}

/* util.py:387  remainder(x - min, max - min) + min, all float32. */
float oracle_wrap(float x, float lo, float hi) {
    float ext = hi - lo;
    float t = x - lo;
    float r = torch_remainder_f(t, ext);
    return r + lo;
}

/* fl32(1e-4 + 1): the Python double 1.0001 as the float32 scalar torch multiplies by. */
static const float H_GROW = 1.00010001659393310546875f;

static float nanmax_f(float a, float b) {
    if (a != a) return a;
    if (b != b) return b;
    return a > b ? a : b;
}

/* util.py:28-79 compute_h, float32 element-wise, torch.max over dims (NaN propagates). */
float oracle_compute_hcell(int dim, const float* qmin, const float* qmax, float hmax, int32_t* cell_count) {
    float ext[3] = {0}, nc[3] = {0}, h[3] = {0};
    int any = 0;
    for (int d = 0; d < dim; ++d) {
        ext[d] = qmax[d] - qmin[d];
        float qc = ext[d] / hmax;
        nc[d] = floorf(qc);
        h[d] = ext[d] / nc[d];
    }
    for (int d = 0; d < dim; ++d) {
        float r = ext[d] / h[d];
        if (r - nc[d] > 0.0f) any = 1;
    }
    if (any) {
        for (int d = 0; d < dim; ++d) {
            nc[d] = nc[d] - 1.0f;
            h[d] = ext[d] / nc[d];
        }
    }
    any = 0;
    for (int d = 0; d < dim; ++d) {
        float r = ext[d] / h[d];
        if (ceilf(r) > r) any = 1;
    }
    if (any)
        for (int d = 0; d < dim; ++d) h[d] = h[d] * H_GROW;
    float hc = h[0];
    for (int d = 1; d < dim; ++d) hc = nanmax_f(hc, h[d]);
    if (cell_count)
        for (int d = 0; d < dim; ++d) cell_count[d] = (int32_t)ceilf(ext[d] / hc); /* cellTable.py:29 */
    return hc;
}

/* hashing.h:20-34 */
int32_t oracle_hash(int dim, const int32_t* c, uint32_t L) {
    if (dim == 1) return (int32_t)(((uint32_t)c[0]) % L);
    static const uint32_t primes[3] = {73856093u, 19349663u, 83492791u};
    uint32_t hsh = 0;
    for (int d = 0; d < dim; ++d) hsh += ((uint32_t)c[d]) * primes[d];
    return (int32_t)(hsh % L);
}

/* neighborhood.h:51-61 / util.py:176-193, int32 wrap-around. */
static int32_t linear_index(int dim, const int32_t* c, const int32_t* cnt) {
    uint32_t lin = 0, prod = 1;
    for (int d = 0; d < dim; ++d) {
        lin += (uint32_t)c[d] * prod;
        prod *= (uint32_t)cnt[d];
    }
    return (int32_t)lin;
}

static int32_t pymod(int32_t n, int32_t m) { return n >= 0 ? n % m : ((n % m) + m) % m; } /* common.h:95-97 */

/* common.h:107-109 moduloOp<float>: float subtraction, the rest in double. */
static double modulo_op(float p, float q, float h) {
    float pq = p - q;
    double half = (double)h / 2.0;
    double t = (double)pq + half;
    return (t - floor(t / (double)h) * (double)h) - half;
}

/* common.h:121-129 modDistance<dim,float> followed by sqrtf. */
static float mod_distance(int dim, const float* xi, const float* xj, const float* dmin, const float* dmax,
                          const uint8_t* periodic) {
    float sum = 0.0f;
    for (int d = 0; d < dim; ++d) {
        double diff;
        if (periodic[d]) diff = modulo_op(xi[d], xj[d], dmax[d] - dmin[d]);
        else diff = (double)(float)(xi[d] - xj[d]);
        sum = (float)((double)sum + diff * diff);
    }
    return sqrtf(sum);
}

static int pair_test(int mode, float dist, float hi, float hj) {
    switch (mode) {
        case OR_SCATTER: return dist < hj;
        case OR_GATHER: return dist < hi;
        case OR_SYMMETRIC: return dist < (hi + hj) / 2.f;
        default: return dist < (hi > hj ? hi : hj); /* std::max(hi, hj) */
    }
}

/* ---------------------------------------------------------------- structure ---- */
typedef struct {
    int dim;
    int64_t nr;
    float hcell;
    int32_t count[3];
    float dmin[3], dmax[3];
    uint8_t periodic[3];
    uint32_t L;
    int64_t* sort_index;   /* [nr] original index of sorted point */
    float* sorted_pos;     /* [nr*dim] */
    float* sorted_sup;     /* [nr] or NULL */
    int64_t ncells;
    int32_t* cell_table;   /* [ncells*3] (lin, begin, count), rows ordered by bucket */
    int32_t* hash_table;   /* [L*2] (first entry, #entries) or (-1, 0) */
} oracle_structure;

typedef struct { int32_t key; int64_t idx; } key_idx;
static int cmp_key_idx(const void* a, const void* b) {
    const key_idx* x = (const key_idx*)a; const key_idx* y = (const key_idx*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

static void cell_of(int dim, const float* x, const float* dmin, float hcell, int32_t* c) {
    for (int d = 0; d < dim; ++d) c[d] = (int32_t)floorf((x[d] - dmin[d]) / hcell);
}

void oracle_structure_free(oracle_structure* s) {
    if (!s) return;
    free(s->sort_index); free(s->sorted_pos); free(s->sorted_sup); free(s->cell_table); free(s->hash_table);
    free(s);
}

/* Build the reference structure over already-wrapped reference positions (hashTable.py:159-234). */
static oracle_structure* build_structure(int dim, int64_t nr, const float* xr, const float* hr, const float* dmin,
                                         const float* dmax, const uint8_t* periodic, float hmax, uint32_t L) {
    oracle_structure* s = (oracle_structure*)calloc(1, sizeof(oracle_structure));
    s->dim = dim; s->nr = nr; s->L = L;
    for (int d = 0; d < dim; ++d) { s->dmin[d] = dmin[d]; s->dmax[d] = dmax[d]; s->periodic[d] = periodic[d]; }
    s->hcell = oracle_compute_hcell(dim, dmin, dmax, hmax, s->count);
    key_idx* ki = (key_idx*)malloc(sizeof(key_idx) * (size_t)(nr > 0 ? nr : 1));
    for (int64_t i = 0; i < nr; ++i) {
        int32_t c[3];
        cell_of(dim, xr + i * dim, dmin, s->hcell, c);
        ki[i].key = linear_index(dim, c, s->count);
        ki[i].idx = i;
    }
    qsort(ki, (size_t)nr, sizeof(key_idx), cmp_key_idx);
    s->sort_index = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nr > 0 ? nr : 1));
    s->sorted_pos = (float*)malloc(sizeof(float) * (size_t)(nr > 0 ? nr * dim : 1));
    s->sorted_sup = hr ? (float*)malloc(sizeof(float) * (size_t)(nr > 0 ? nr : 1)) : NULL;
    int64_t ncells = 0;
    for (int64_t i = 0; i < nr; ++i) {
        s->sort_index[i] = ki[i].idx;
        memcpy(s->sorted_pos + i * dim, xr + ki[i].idx * dim, sizeof(float) * dim);
        if (hr) s->sorted_sup[i] = hr[ki[i].idx];
        if (i == 0 || ki[i].key != ki[i - 1].key) ++ncells;
    }
    /* unique_consecutive runs -> (lin, begin, count); coordinates of a run's first point. */
    int32_t* cells = (int32_t*)malloc(sizeof(int32_t) * 3 * (size_t)(ncells > 0 ? ncells : 1));
    key_idx* bucket = (key_idx*)malloc(sizeof(key_idx) * (size_t)(ncells > 0 ? ncells : 1));
    int64_t ci = -1;
    for (int64_t i = 0; i < nr; ++i) {
        if (i == 0 || ki[i].key != ki[i - 1].key) {
            ++ci;
            cells[ci * 3 + 0] = ki[i].key;
            cells[ci * 3 + 1] = (int32_t)i;
            cells[ci * 3 + 2] = 0;
            int32_t c[3];
            cell_of(dim, s->sorted_pos + i * dim, dmin, s->hcell, c); /* hashTable.py:201-202 */
            bucket[ci].key = oracle_hash(dim, c, L);
            bucket[ci].idx = ci;
        }
        cells[ci * 3 + 2] += 1;
    }
    free(ki);
    qsort(bucket, (size_t)ncells, sizeof(key_idx), cmp_key_idx);
    s->ncells = ncells;
    s->cell_table = (int32_t*)malloc(sizeof(int32_t) * 3 * (size_t)(ncells > 0 ? ncells : 1));
    s->hash_table = (int32_t*)malloc(sizeof(int32_t) * 2 * (size_t)L);
    for (uint32_t b = 0; b < L; ++b) { s->hash_table[2 * b] = -1; s->hash_table[2 * b + 1] = 0; }
    for (int64_t k = 0; k < ncells; ++k) {
        memcpy(s->cell_table + 3 * k, cells + 3 * bucket[k].idx, sizeof(int32_t) * 3);
        int32_t b = bucket[k].key;
        if (s->hash_table[2 * b] < 0) s->hash_table[2 * b] = (int32_t)k;
        s->hash_table[2 * b + 1] += 1;
    }
    free(cells); free(bucket);
    return s;
}

/* neighborhood.h:73-96 queryHashMap */
static int lookup(const oracle_structure* s, const int32_t* cell, int32_t* begin, int32_t* end) {
    int32_t lin = linear_index(s->dim, cell, s->count);
    int32_t b = oracle_hash(s->dim, cell, s->L);
    int32_t hb = s->hash_table[2 * b], hl = s->hash_table[2 * b + 1];
    if (hb == -1) return 0;
    for (int32_t i = hb; i < hb + hl; ++i) {
        if (s->cell_table[3 * i] == lin) {
            *begin = s->cell_table[3 * i + 1];
            *end = *begin + s->cell_table[3 * i + 2];
            return 1;
        }
    }
    return 0;
}

/* Visit every candidate of query position xi (neighborhoodDynamic.h:37-115).  When out is
 * NULL only counts; otherwise writes original reference indices. */
static int64_t search_one(const oracle_structure* s, int mode, const float* xi, float hi, int64_t* out) {
    int dim = s->dim;
    int32_t qc[3];
    cell_of(dim, xi, s->dmin, s->hcell, qc);
    int nofs = 1;
    for (int d = 0; d < dim; ++d) nofs *= 3;
    int64_t n = 0;
    for (int o = 0; o < nofs; ++o) {
        int32_t cell[3];
        int rem = o;
        for (int d = dim - 1; d >= 0; --d) { /* last coordinate fastest */
            int32_t off = rem % 3 - 1;
            rem /= 3;
            cell[d] = s->periodic[d] ? pymod(qc[d] + off, s->count[d]) : qc[d] + off;
        }
        int32_t b, e;
        if (!lookup(s, cell, &b, &e)) continue;
        for (int32_t j = b; j < e; ++j) {
            float dist = mod_distance(dim, xi, s->sorted_pos + (int64_t)j * dim, s->dmin, s->dmax, s->periodic);
            float hj = s->sorted_sup ? s->sorted_sup[j] : 0.0f;
            if (pair_test(mode, dist, hi, hj)) {
                if (out) out[n] = s->sort_index[j];
                ++n;
            }
        }
    }
    return n;
}

/* ------------------------------------------------------------------ results ---- */
typedef struct {
    int64_t nq, npairs;
    int64_t* counts;  /* [nq]   rowEntries */
    int64_t* offsets; /* [nq+1] */
    int64_t* col;     /* [npairs] original reference index, rows in query order */
    float hcell;
    int32_t count[3];
    int status;       /* 0 ok, <0 error */
} oracle_result;

void oracle_result_free(oracle_result* r) {
    if (!r) return;
    free(r->counts); free(r->offsets); free(r->col); free(r);
}

static float max_f(const float* v, int64_t n) {
    float m = -INFINITY;
    for (int64_t i = 0; i < n; ++i) m = nanmax_f(m, v[i]);
    return m;
}

/*
 * Full radiusSearch(..., algorithm='compact') with an explicit DomainDescription
 * (neighborhood.py:136-309 -> compactSearch.py:12-171 -> cppSearch.py:179-244).
 * xq/xr are the caller's raw positions; the wraps the reference applies are applied here.
 * hq may be NULL for scatter, hr may be NULL for gather.  hashMapLength > 0.
 */
oracle_result* oracle_radius_search(int dim, int64_t nq, const float* xq, const float* hq, int64_t nr,
                                    const float* xr, const float* hr, const float* dmin, const float* dmax,
                                    const uint8_t* periodic, int mode, int64_t hash_map_length) {
    oracle_result* r = (oracle_result*)calloc(1, sizeof(oracle_result));
    r->nq = nq;
    if (dim < 1 || dim > 3 || hash_map_length <= 0) { r->status = -1; return r; }
    /* wraps: queries once (radiusSearch), references twice (radiusSearch + neighborSearch_cpp) */
    float* wq = (float*)malloc(sizeof(float) * (size_t)(nq * dim > 0 ? nq * dim : 1));
    float* wr = (float*)malloc(sizeof(float) * (size_t)(nr * dim > 0 ? nr * dim : 1));
    for (int64_t i = 0; i < nq; ++i)
        for (int d = 0; d < dim; ++d) {
            float v = xq[i * dim + d];
            wq[i * dim + d] = periodic[d] ? oracle_wrap(v, dmin[d], dmax[d]) : v;
        }
    for (int64_t i = 0; i < nr; ++i)
        for (int d = 0; d < dim; ++d) {
            float v = xr[i * dim + d];
            wr[i * dim + d] = periodic[d] ? oracle_wrap(oracle_wrap(v, dmin[d], dmax[d]), dmin[d], dmax[d]) : v;
        }
    /* cellTable.py:40-81 computeGridSupport */
    float hmax;
    if (mode == OR_SCATTER) hmax = max_f(hr, nr);
    else if (mode == OR_GATHER) hmax = max_f(hq, nq);
    else hmax = nanmax_f(max_f(hr, nr), max_f(hq, nq));
    oracle_structure* s = build_structure(dim, nr, wr, hr, dmin, dmax, periodic, hmax, (uint32_t)hash_map_length);
    r->hcell = s->hcell;
    for (int d = 0; d < dim; ++d) r->count[d] = s->count[d];
    for (int d = 0; d < dim; ++d)
        if (periodic[d] && s->count[d] <= 0) { r->status = -2; oracle_structure_free(s); free(wq); free(wr); return r; }
    r->counts = (int64_t*)calloc((size_t)(nq > 0 ? nq : 1), sizeof(int64_t));
    r->offsets = (int64_t*)calloc((size_t)nq + 1, sizeof(int64_t));
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < nq; ++i)
        r->counts[i] = search_one(s, mode, wq + i * dim, hq ? hq[i] : 0.0f, NULL);
    for (int64_t i = 0; i < nq; ++i) r->offsets[i + 1] = r->offsets[i] + r->counts[i];
    r->npairs = r->offsets[nq];
    r->col = (int64_t*)malloc(sizeof(int64_t) * (size_t)(r->npairs > 0 ? r->npairs : 1));
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < nq; ++i)
        search_one(s, mode, wq + i * dim, hq ? hq[i] : 0.0f, r->col + r->offsets[i]);
    oracle_structure_free(s);
    free(wq); free(wr);
    return r;
}

/* All-pairs version of the same test with the same wraps and no grid: the pair set the
 * compact search returns whenever its grid visits every pair inside the support. */
oracle_result* oracle_brute_force(int dim, int64_t nq, const float* xq, const float* hq, int64_t nr,
                                  const float* xr, const float* hr, const float* dmin, const float* dmax,
                                  const uint8_t* periodic, int mode) {
    oracle_result* r = (oracle_result*)calloc(1, sizeof(oracle_result));
    r->nq = nq;
    float* wq = (float*)malloc(sizeof(float) * (size_t)(nq * dim > 0 ? nq * dim : 1));
    float* wr = (float*)malloc(sizeof(float) * (size_t)(nr * dim > 0 ? nr * dim : 1));
    for (int64_t i = 0; i < nq; ++i)
        for (int d = 0; d < dim; ++d) {
            float v = xq[i * dim + d];
            wq[i * dim + d] = periodic[d] ? oracle_wrap(v, dmin[d], dmax[d]) : v;
        }
    for (int64_t i = 0; i < nr; ++i)
        for (int d = 0; d < dim; ++d) {
            float v = xr[i * dim + d];
            wr[i * dim + d] = periodic[d] ? oracle_wrap(oracle_wrap(v, dmin[d], dmax[d]), dmin[d], dmax[d]) : v;
        }
    r->counts = (int64_t*)calloc((size_t)(nq > 0 ? nq : 1), sizeof(int64_t));
    r->offsets = (int64_t*)calloc((size_t)nq + 1, sizeof(int64_t));
    for (int pass = 0; pass < 2; ++pass) {
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t i = 0; i < nq; ++i) {
            int64_t n = 0;
            for (int64_t j = 0; j < nr; ++j) {
                float dist = mod_distance(dim, wq + i * dim, wr + j * dim, dmin, dmax, periodic);
                if (pair_test(mode, dist, hq ? hq[i] : 0.0f, hr ? hr[j] : 0.0f)) {
                    if (pass) r->col[r->offsets[i] + n] = j;
                    ++n;
                }
            }
            if (!pass) r->counts[i] = n;
        }
        if (!pass) {
            for (int64_t i = 0; i < nq; ++i) r->offsets[i + 1] = r->offsets[i] + r->counts[i];
            r->npairs = r->offsets[nq];
            r->col = (int64_t*)malloc(sizeof(int64_t) * (size_t)(r->npairs > 0 ? r->npairs : 1));
        }
    }
    free(wq); free(wr);
    return r;
}

/* Accessors for ctypes callers. */
int oracle_result_status(const oracle_result* r) { return r->status; }
int64_t oracle_result_npairs(const oracle_result* r) { return r->npairs; }
float oracle_result_hcell(const oracle_result* r) { return r->hcell; }
void oracle_result_cell_count(const oracle_result* r, int32_t* out3) { memcpy(out3, r->count, sizeof(r->count)); }
void oracle_result_copy(const oracle_result* r, int64_t* counts, int64_t* col) {
    if (counts && r->nq) memcpy(counts, r->counts, sizeof(int64_t) * (size_t)r->nq);
    if (col && r->npairs) memcpy(col, r->col, sizeof(int64_t) * (size_t)r->npairs);
}
int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
