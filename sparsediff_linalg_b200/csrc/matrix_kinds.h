// Private layouts of the three matrix kinds behind the upstream `matrix` handle
// (upstream src/internal/sparse_matrix.h:32-54, permuted_dense.h:29-78,
// stacked_pd.h:28-54). Each embeds the handle first so a matrix* is a pointer to the
// kind; the device-side state lives in a C++ object the kind points to.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "capi_common.h"
#include "sparsediff_linalg/matrix.h"

namespace sdl {

// Device copy of a compressed structure, shared by every plan that reads it so
// the structure outlives whichever matrix handle is freed first.
struct DevStruct
{
    int rows = 0, cols = 0, nnz = 0;
    DevBuf<int> p, i;
};

// Device copy of a value array, refreshed iff the owner's values_version moved.
struct DevValues
{
    DevBuf<double> x;
    uint64_t seen = 0;
    bool valid = false;
};

struct BoundOp
{
    virtual ~BoundOp() = default;
};

struct SparseImpl
{
    std::shared_ptr<DevStruct> st;              // device CSR structure (lazy)
    DevValues vals;                             // device CSR values
    std::shared_ptr<TransposePlan> csc;         // device CSC mirror structure + CSR positions
    std::unique_ptr<BoundOp> bound;             // state bound by the alloc that produced it
};

struct PdImpl;
struct SpdImpl;

} // namespace sdl

struct sdl_sparse
{
    matrix base;
    CSR_matrix *csr;
    sdl::SparseImpl *impl;
};

// permuted_dense: M[row_perm[ii], col_perm[jj]] = X[ii * n0 + jj].
struct permuted_dense
{
    matrix base;
    int m0, n0;
    int *row_perm, *col_perm;
    int *row_inv, *col_inv; // -1 outside the perms
    double *X;
    bool owns_X;
    CSR_matrix *csr_cache; // to_csr view; x aliases X
    sdl::PdImpl *impl;
};

struct sdl_stacked
{
    matrix base;
    int n_blocks;
    permuted_dense **blocks;
    int *src_block_idx_p, *src_block_idx;
    double *values; // shared value buffer (block-major)
    CSR_matrix *csr_cache;
    sdl::SpdImpl *impl;
};

namespace sdl {

inline sdl_sparse *as_sparse(const matrix *m) { return (sdl_sparse *)m; }
inline permuted_dense *as_pd(const matrix *m) { return (permuted_dense *)m; }
inline sdl_stacked *as_spd(const matrix *m) { return (sdl_stacked *)m; }

// sparse kind helpers shared with the dense-kind file
const DevStruct &sparse_dev_struct(sdl_sparse *A, cudaStream_t s);
const double *sparse_dev_values(sdl_sparse *A, cudaStream_t s);
const TransposePlan &sparse_dev_csc(sdl_sparse *A, cudaStream_t s);
matrix *sparse_wrap(CSR_matrix *csr);
// Copy the device values of a sparse output into its host CSR and publish them
// (version bumped, device copy marked fresh).
void publish_output(sdl_sparse *C, cudaStream_t s);
// New sparse output whose structure is (Cp, Ci) on the device; host copy made.
sdl_sparse *new_output(int m, int n, int nnz, const int *d_Cp, const int *d_Ci, cudaStream_t s);

// dense kinds (capi_dense.cpp)
void pd_free(permuted_dense *pd);
void spd_free(sdl_stacked *spd);
matrix *pd_copy_sparsity(const permuted_dense *A);
matrix *spd_copy_sparsity(const sdl_stacked *A);
matrix *dense_BTA_alloc(matrix *A, matrix *B);
void dense_BTDA_fill(matrix *A, const double *d, matrix *B, matrix *C);
matrix *dense_BA_alloc(const matrix *B, matrix *A);
void dense_BA_fill(const matrix *B, const matrix *A, matrix *C);
matrix *dense_ATA_alloc(matrix *A);
void dense_ATDA_fill(const matrix *A, const double *d, matrix *C);
void dense_DA_fill(const double *d, const matrix *A, matrix *C);
matrix *dense_transpose_alloc(const matrix *A);
void dense_transpose_fill(const matrix *A, matrix *AT);

} // namespace sdl
