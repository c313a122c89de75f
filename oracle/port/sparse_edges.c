/*
 * CPU restatement of the MATLAB-side steps around the element kernels.
 * TEST INFRASTRUCTURE ONLY (results to compare the GPU with; see oracle.h).
 *   oracle_generate_edges  src/Mesh.m:114-138
 *   oracle_sparse_csr      MATLAB sparse() as called at src/Assembler.m:37-38, 205-206
 *   oracle_sparse_vec      src/Assembler.m:211-216
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

/* ---- Mesh.generateEdges ------------------------------------------------- */

typedef struct {
    int32_t lo, hi;
    int64_t slot; /* 6*e + k */
} edge_rec;

static int cmp_edge(const void *a, const void *b) {
    const edge_rec *x = (const edge_rec *)a, *y = (const edge_rec *)b;
    if (x->lo != y->lo) return x->lo < y->lo ? -1 : 1;
    if (x->hi != y->hi) return x->hi < y->hi ? -1 : 1;
    return (x->slot > y->slot) - (x->slot < y->slot);
}

int64_t oracle_generate_edges(const int32_t *T, int64_t Ne, int32_t *edges_out, int64_t edges_cap,
                              int32_t *t2e, int8_t *sign) {
    /* local edge table (1,2),(1,3),(1,4),(2,3),(2,4),(3,4): Mesh.m:118 */
    static const int ends[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
    int64_t n = 6 * Ne;
    edge_rec *r = (edge_rec *)malloc((size_t)(n ? n : 1) * sizeof(edge_rec));
    if (!r) return -1;
    for (int64_t e = 0; e < Ne; e++)
        for (int k = 0; k < 6; k++) {
            int32_t s = T[4 * e + ends[k][0]], t = T[4 * e + ends[k][1]];
            edge_rec *x = &r[6 * e + k];
            x->lo = s < t ? s : t;
            x->hi = s < t ? t : s;
            x->slot = 6 * e + k;
            /* +1 iff the local start node is the smaller global id (:134-135) */
            sign[6 * e + k] = (int8_t)(s < t ? 1 : -1);
        }
    /* unique(sort(rows)) numbers edges lexicographically by (min,max) (:126-128) */
    qsort(r, (size_t)n, sizeof(edge_rec), cmp_edge);
    int64_t E = 0;
    for (int64_t i = 0; i < n; i++) {
        if (i == 0 || r[i].lo != r[i - 1].lo || r[i].hi != r[i - 1].hi) {
            if (E < edges_cap) {
                edges_out[2 * E] = r[i].lo;
                edges_out[2 * E + 1] = r[i].hi;
            }
            E++;
        }
        t2e[r[i].slot] = (int32_t)E; /* 1-based, like ic */
    }
    free(r);
    return E;
}

/* ---- sparse(I,J,V,N,N) -------------------------------------------------- */

int64_t oracle_sparse_csr(const double *I, const double *J, const double *V, int64_t n, int64_t N,
                          int drop_zeros, int64_t *row_ptr, int32_t *col_idx, double *vals) {
    /* Stable two-pass counting sort: by column, then by row. Entries with equal
     * (row, col) keep their order of appearance and are summed in that order. */
    int64_t *cnt = (int64_t *)calloc((size_t)N + 2, sizeof(int64_t));
    int64_t *tmp = (int64_t *)malloc((size_t)(n ? n : 1) * sizeof(int64_t));
    int64_t *ord = (int64_t *)malloc((size_t)(n ? n : 1) * sizeof(int64_t));
    if (!cnt || !tmp || !ord) {
        free(cnt);
        free(tmp);
        free(ord);
        return -1;
    }
    int64_t m = 0;
    for (int64_t t = 0; t < n; t++) {
        if (!(I[t] > 0 && J[t] > 0)) continue; /* valid mask, Assembler.m:37 */
        if (I[t] > (double)N || J[t] > (double)N) {
            free(cnt);
            free(tmp);
            free(ord);
            return -1;
        }
        cnt[(int64_t)J[t]]++;
        m++;
    }
    for (int64_t c = 1; c <= N + 1; c++) cnt[c] += cnt[c - 1];
    for (int64_t t = 0; t < n; t++) {
        if (!(I[t] > 0 && J[t] > 0)) continue;
        int64_t c = (int64_t)J[t] - 1;
        tmp[cnt[c]++] = t;
    }
    memset(cnt, 0, ((size_t)N + 2) * sizeof(int64_t));
    for (int64_t u = 0; u < m; u++) cnt[(int64_t)I[tmp[u]]]++;
    for (int64_t r = 1; r <= N + 1; r++) cnt[r] += cnt[r - 1];
    for (int64_t u = 0; u < m; u++) {
        int64_t r = (int64_t)I[tmp[u]] - 1;
        ord[cnt[r]++] = tmp[u];
    }
    /* ord is sorted by (row, col), stable; sum runs of equal keys */
    int64_t nnz = 0;
    int64_t u = 0;
    if (row_ptr) row_ptr[0] = 0;
    int64_t cur_row = 0;
    while (u < m) {
        int64_t t0 = ord[u];
        int64_t r = (int64_t)I[t0] - 1, c = (int64_t)J[t0] - 1;
        double s = V[t0];
        int64_t w = u + 1;
        while (w < m && (int64_t)I[ord[w]] - 1 == r && (int64_t)J[ord[w]] - 1 == c) {
            s += V[ord[w]];
            w++;
        }
        if (!(drop_zeros && s == 0.0)) {
            if (col_idx) {
                while (cur_row < r) row_ptr[++cur_row] = nnz;
                col_idx[nnz] = (int32_t)c;
                vals[nnz] = s;
            }
            nnz++;
        }
        u = w;
    }
    if (col_idx)
        while (cur_row < N) row_ptr[++cur_row] = nnz;
    free(cnt);
    free(tmp);
    free(ord);
    return nnz;
}

int oracle_sparse_vec(const double *Ridx, const double *Rval, int64_t n, int64_t N, double *out) {
    memset(out, 0, (size_t)N * sizeof(double));
    for (int64_t t = 0; t < n; t++) {
        if (!(Ridx[t] > 0)) continue; /* valid_r, Assembler.m:214 */
        int64_t r = (int64_t)Ridx[t] - 1;
        if (r >= N) return -1;
        out[r] += Rval[t];
    }
    return 0;
}
