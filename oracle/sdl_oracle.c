/* CPU oracle (test infrastructure only; never linked into the product library).
 *
 * Plain-C restatement of the upstream sparse-product algorithms. Each function
 * cites the upstream source it follows (paths relative to the upstream project)
 * and keeps its visiting order and roundings: products are formed as
 * (L.x * d[k]) * A.x and accumulated with += from +0.0, with no FMA (this file is
 * built without -march, like upstream). */
#include "sdl_oracle.h"

#include <stdlib.h>
#include <string.h>

static int cmp_int(const void *a, const void *b)
{
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

/* src/sparse/gustavson.c:26-68 (pass 1): the number of distinct columns of every
 * row of C, using a "last row that saw column j" stamp. */
long long orc_gustavson_count(const int *Lp, const int *Li, int L_m, int blocks,
                              const int *Ap, const int *Ai, int A_m, int A_n, int *Cp,
                              int *work)
{
    int n_L = A_m / blocks;
    int *stamp = work;
    for (int j = 0; j < A_n; ++j) stamp[j] = -1;
    long long total = 0;
    Cp[0] = 0;
    for (int b = 0; b < blocks; ++b)
        for (int r = 0; r < L_m; ++r)
        {
            int row = b * L_m + r;
            int cnt = 0;
            for (int ii = Lp[r]; ii < Lp[r + 1]; ++ii)
            {
                int k = Li[ii] + b * n_L;
                for (int jj = Ap[k]; jj < Ap[k + 1]; ++jj)
                {
                    int j = Ai[jj];
                    if (stamp[j] != row)
                    {
                        stamp[j] = row;
                        ++cnt;
                    }
                }
            }
            total += cnt;
            if (total > 2147483647LL) return -1;
            Cp[row + 1] = (int)total;
        }
    return total;
}

/* src/sparse/gustavson.c:70-102 (pass 2): emit each row's distinct columns in
 * first-seen order, then sort the row ascending (upstream qsorts it). */
void orc_gustavson_structure(const int *Lp, const int *Li, int L_m, int blocks,
                             const int *Ap, const int *Ai, int A_m, int A_n,
                             const int *Cp, int *Ci, int *work)
{
    int n_L = A_m / blocks;
    int *stamp = work;
    for (int j = 0; j < A_n; ++j) stamp[j] = -1;
    for (int b = 0; b < blocks; ++b)
        for (int r = 0; r < L_m; ++r)
        {
            int row = b * L_m + r;
            int at = Cp[row];
            for (int ii = Lp[r]; ii < Lp[r + 1]; ++ii)
            {
                int k = Li[ii] + b * n_L;
                for (int jj = Ap[k]; jj < Ap[k + 1]; ++jj)
                {
                    int j = Ai[jj];
                    if (stamp[j] != row)
                    {
                        stamp[j] = row;
                        Ci[at++] = j;
                    }
                }
            }
            if (Cp[row + 1] - Cp[row] > 1)
                qsort(Ci + Cp[row], (size_t)(Cp[row + 1] - Cp[row]), sizeof(int), cmp_int);
        }
}

/* src/sparse/gustavson.c:107-143: dense accumulator, zeroed on the row's pattern,
 * acc[j] += (L.x[ii] * d[k]) * A.x[jj] over ii in L-row order then jj, gathered
 * back in C's column order. */
void orc_gustavson_values(const int *Lp, const int *Li, const double *Lx, int L_m,
                          int blocks, const double *d, const int *Ap, const int *Ai,
                          const double *Ax, int A_m, int A_n, const int *Cp,
                          const int *Ci, double *Cx, double *work)
{
    int n_L = A_m / blocks;
    double *acc = work;
    (void)A_n;
    for (int b = 0; b < blocks; ++b)
        for (int r = 0; r < L_m; ++r)
        {
            int row = b * L_m + r;
            for (int q = Cp[row]; q < Cp[row + 1]; ++q) acc[Ci[q]] = 0.0;
            for (int ii = Lp[r]; ii < Lp[r + 1]; ++ii)
            {
                int k = Li[ii] + b * n_L;
                double lv = Lx ? Lx[ii] : 1.0;
                double v = d ? lv * d[k] : lv;
                for (int jj = Ap[k]; jj < Ap[k + 1]; ++jj) acc[Ai[jj]] += v * Ax[jj];
            }
            for (int q = Cp[row]; q < Cp[row + 1]; ++q) Cx[q] = acc[Ci[q]];
        }
}

/* src/sparse/CSC_matrix.c:62-123 (and CSR_matrix.c:99-142): count per column,
 * exclusive scan, scatter in row-major order, so source rows stay ascending
 * inside every output row. */
void orc_transpose(const int *p, const int *idx, const double *x, int rows, int cols,
                   int *Tp, int *Ti, double *Tx, int *work)
{
    int *next = work;
    memset(next, 0, (size_t)cols * sizeof(int));
    for (int e = 0; e < p[rows]; ++e) next[idx[e]]++;
    Tp[0] = 0;
    for (int c = 0; c < cols; ++c)
    {
        Tp[c + 1] = Tp[c] + next[c];
        next[c] = Tp[c];
    }
    for (int r = 0; r < rows; ++r)
        for (int e = p[r]; e < p[r + 1]; ++e)
        {
            int at = next[idx[e]]++;
            Ti[at] = r;
            if (x && Tx) Tx[at] = x[e];
        }
}

/* Coalescing has no upstream function; its semantics are upstream's row_reduce
 * (src/sparse/sparse_matrix.c:136-240) applied to the CSR with one triplet per row
 * and group[t] = rows[t]: sources of an output row taken in ascending t (the
 * counting sort of :146-164), the row's columns sorted (:198-201), and values
 * summed from +0.0 in ascending source order (accumulator, src/sparse/CSR_sum.c:150-157). */
static void coalesce_group(const int *rows, int nnz, int m, int *start, int *order)
{
    memset(start, 0, ((size_t)m + 1) * sizeof(int));
    for (int t = 0; t < nnz; ++t) start[rows[t] + 1]++;
    for (int r = 0; r < m; ++r) start[r + 1] += start[r];
    int *fill = (int *)malloc(((size_t)m + 1) * sizeof(int));
    memcpy(fill, start, ((size_t)m + 1) * sizeof(int));
    for (int t = 0; t < nnz; ++t) order[fill[rows[t]]++] = t;
    free(fill);
}

long long orc_coalesce_count(const int *rows, const int *cols, int nnz, int m, int n,
                             int *Cp)
{
    int *start = (int *)malloc(((size_t)m + 1) * sizeof(int));
    int *order = (int *)malloc(((size_t)nnz + 1) * sizeof(int));
    int *stamp = (int *)malloc(((size_t)n + 1) * sizeof(int));
    coalesce_group(rows, nnz, m, start, order);
    for (int j = 0; j < n; ++j) stamp[j] = -1;
    long long total = 0;
    Cp[0] = 0;
    for (int r = 0; r < m; ++r)
    {
        for (int s = start[r]; s < start[r + 1]; ++s)
        {
            int j = cols[order[s]];
            if (stamp[j] != r)
            {
                stamp[j] = r;
                ++total;
            }
        }
        Cp[r + 1] = (int)total;
    }
    free(start);
    free(order);
    free(stamp);
    return total;
}

void orc_coalesce_fill(const int *rows, const int *cols, const double *x, int nnz, int m,
                       int n, const int *Cp, int *Ci, double *Cx)
{
    int *start = (int *)malloc(((size_t)m + 1) * sizeof(int));
    int *order = (int *)malloc(((size_t)nnz + 1) * sizeof(int));
    int *stamp = (int *)malloc(((size_t)n + 1) * sizeof(int));
    int *pos = (int *)malloc(((size_t)n + 1) * sizeof(int));
    coalesce_group(rows, nnz, m, start, order);
    for (int j = 0; j < n; ++j) stamp[j] = -1;
    for (int r = 0; r < m; ++r)
    {
        int at = Cp[r];
        for (int s = start[r]; s < start[r + 1]; ++s)
        {
            int j = cols[order[s]];
            if (stamp[j] != r)
            {
                stamp[j] = r;
                Ci[at++] = j;
            }
        }
        if (Cp[r + 1] - Cp[r] > 1)
            qsort(Ci + Cp[r], (size_t)(Cp[r + 1] - Cp[r]), sizeof(int), cmp_int);
        for (int q = Cp[r]; q < Cp[r + 1]; ++q)
        {
            pos[Ci[q]] = q;
            Cx[q] = 0.0;
        }
        for (int s = start[r]; s < start[r + 1]; ++s)
        {
            int t = order[s];
            Cx[pos[cols[t]]] += x[t];
        }
    }
    free(start);
    free(order);
    free(stamp);
    free(pos);
}

/* src/sparse/sparse_matrix.c:79-134: C's row i is a copy of A's row map[i]. */
long long orc_row_gather_count(const int *Ap, const int *map, int m_out, int *Cp)
{
    long long total = 0;
    Cp[0] = 0;
    for (int i = 0; i < m_out; ++i)
    {
        total += Ap[map[i] + 1] - Ap[map[i]];
        if (total > 2147483647LL) return -1;
        Cp[i + 1] = (int)total;
    }
    return total;
}

void orc_row_gather_fill(const int *Ap, const int *Ai, const double *Ax, const int *map,
                         int m_out, const int *Cp, int *Ci, double *Cx)
{
    for (int i = 0; i < m_out; ++i)
    {
        int len = Cp[i + 1] - Cp[i];
        memcpy(Ci + Cp[i], Ai + Ap[map[i]], (size_t)len * sizeof(int));
        memcpy(Cx + Cp[i], Ax + Ap[map[i]], (size_t)len * sizeof(double));
    }
}

/* src/sparse/sparse_matrix.c:136-240: group the source rows by output row
 * (ascending source row), sorted union of their columns, then every source entry
 * added in ascending source position into a zeroed output. */
long long orc_row_reduce_count(const int *Ap, const int *Ai, int m, int n,
                               const int *group, int m_out, int *Cp)
{
    int *start = (int *)malloc(((size_t)m_out + 1) * sizeof(int));
    int *order = (int *)malloc(((size_t)m + 1) * sizeof(int));
    int *stamp = (int *)malloc(((size_t)n + 1) * sizeof(int));
    coalesce_group(group, m, m_out, start, order);
    for (int j = 0; j < n; ++j) stamp[j] = -1;
    long long total = 0;
    Cp[0] = 0;
    for (int g = 0; g < m_out; ++g)
    {
        for (int s = start[g]; s < start[g + 1]; ++s)
        {
            int i = order[s];
            for (int e = Ap[i]; e < Ap[i + 1]; ++e)
                if (stamp[Ai[e]] != g)
                {
                    stamp[Ai[e]] = g;
                    ++total;
                }
        }
        Cp[g + 1] = (int)total;
    }
    free(start);
    free(order);
    free(stamp);
    return total;
}

void orc_row_reduce_fill(const int *Ap, const int *Ai, const double *Ax, int m, int n,
                         const int *group, int m_out, const int *Cp, int *Ci,
                         double *Cx)
{
    int *start = (int *)malloc(((size_t)m_out + 1) * sizeof(int));
    int *order = (int *)malloc(((size_t)m + 1) * sizeof(int));
    int *stamp = (int *)malloc(((size_t)n + 1) * sizeof(int));
    int *pos = (int *)malloc(((size_t)n + 1) * sizeof(int));
    coalesce_group(group, m, m_out, start, order);
    for (int j = 0; j < n; ++j) stamp[j] = -1;
    for (int g = 0; g < m_out; ++g)
    {
        int at = Cp[g];
        for (int s = start[g]; s < start[g + 1]; ++s)
        {
            int i = order[s];
            for (int e = Ap[i]; e < Ap[i + 1]; ++e)
                if (stamp[Ai[e]] != g)
                {
                    stamp[Ai[e]] = g;
                    Ci[at++] = Ai[e];
                }
        }
        if (Cp[g + 1] - Cp[g] > 1)
            qsort(Ci + Cp[g], (size_t)(Cp[g + 1] - Cp[g]), sizeof(int), cmp_int);
    }
    for (int q = 0; q < Cp[m_out]; ++q) Cx[q] = 0.0;
    /* ascending source position e == ascending (source row, position in row) */
    for (int i = 0; i < m; ++i)
    {
        int g = group[i];
        for (int q = Cp[g]; q < Cp[g + 1]; ++q) pos[Ci[q]] = q;
        for (int e = Ap[i]; e < Ap[i + 1]; ++e) Cx[pos[Ai[e]]] += Ax[e];
    }
    free(start);
    free(order);
    free(stamp);
    free(pos);
}

void orc_dense_btdb(const double *A, const double *B, const double *w, int K, int rows,
                    int cols, double *C)
{
    for (int r = 0; r < rows; ++r)
        for (int c = 0; c < cols; ++c)
        {
            double s = 0.0;
            for (int k = 0; k < K; ++k)
            {
                double a = A[(size_t)k * rows + r];
                double t = w ? a * w[k] : a;
                s += t * B[(size_t)k * cols + c];
            }
            C[(size_t)r * cols + c] = s;
        }
}
