// Upstream-compatible raw entry points (CSR_matrix.h, CSC_matrix.h, COO_matrix.h)
// on host structs, computed on the GPU.
//
// Each *_alloc runs the symbolic phase on the device and binds the device-side
// plan (operand structures, numeric schedule, value buffers) to the output object
// it returns; the matching *_fill_values finds that plan, uploads the operand
// values, runs the numeric kernels and downloads the result. Fills make no device
// allocation. A plan is dropped when its output is freed through this library;
// every lookup also checks the output's shape and arrays, so an object freed some
// other way can never be matched by a later one at the same address.
#include <climits>
#include <memory>
#include <mutex>
#include <unordered_map>

#include "capi_common.h"
#include "sparsediff_linalg/COO_matrix.h"
#include "sparsediff_linalg/CSC_matrix.h"
#include "sparsediff_linalg/CSR_matrix.h"
#include "sparsediff_linalg/tracked_alloc.h"

// The tracked-allocation counters are always present so the symbols exist whichever
// way a consumer sets SP_TRACK_MEMORY (the library itself never allocates through
// the inline sp_* wrappers of a tracking consumer).
extern "C" {
size_t g_allocated_bytes = 0;
size_t g_peak_bytes = 0;
void sp_memory_stats(size_t *live_bytes, size_t *peak_bytes)
{
    if (live_bytes) *live_bytes = g_allocated_bytes;
    if (peak_bytes) *peak_bytes = g_peak_bytes;
}
void sp_memory_reset_peak(void) { g_peak_bytes = g_allocated_bytes; }
}

namespace sdl {

// ------------------------------------------------------------------ status
static thread_local sdl_status t_status = SDL_OK;
static thread_local std::string t_message;
static std::atomic<int> g_fatal{1};

void set_status(sdl_status code, const std::string &msg)
{
    t_status = code;
    t_message = msg;
}
bool fatal_errors() { return g_fatal.load() != 0; }

void check_device_errors(cudaStream_t s, const char *what)
{
    int e = take_device_error(s);
    if (e)
        fail(SDL_ERR_INTERNAL, std::string(what) + ": device-side consistency check failed "
                                                   "(operand structure changed after alloc?)");
}

// ------------------------------------------------------------------ plans
namespace {

struct Key
{
    const void *obj;
    int m, n, nnz;
    const void *p, *i;
};

struct RawPlan
{
    Key key{};
    virtual ~RawPlan() = default;
};

struct ProductPlan : RawPlan
{
    int A_m = 0, A_n = 0, A_nnz = 0, B_m = 0, B_n = 0, B_nnz = 0;
    DevBuf<int> Ap, Ai, Lp, Li;
    Product P;
    DevBuf<double> Lx, Ax, dv, Cx;
};

struct TransposeRawPlan : RawPlan
{
    int rows = 0, cols = 0, nnz = 0;
    TransposePlan T;
    DevBuf<double> x, Tx;
};

struct CoalesceRawPlan : RawPlan
{
    int m = 0, n = 0, nnz_in = 0;
    DevBuf<int> rows, cols;
    sdl_coalesce *plan = nullptr;
    DevBuf<double> x, Cx;
    ~CoalesceRawPlan() override { sdl_coalesce_destroy(plan); }
};

std::mutex g_mu;
std::unordered_map<const void *, std::unique_ptr<RawPlan>> g_plans;

template <class S>
Key key_of(const S *obj)
{
    return Key{obj, obj->m, obj->n, obj->nnz, obj->p, obj->i};
}

void put_plan(std::unique_ptr<RawPlan> plan)
{
    std::lock_guard<std::mutex> lk(g_mu);
    const void *k = plan->key.obj;
    g_plans[k] = std::move(plan);
}

template <class PlanT, class S>
PlanT *find_plan(const S *obj)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_plans.find(obj);
    if (it == g_plans.end()) return nullptr;
    Key k = key_of(obj);
    const Key &s = it->second->key;
    if (s.m != k.m || s.n != k.n || s.nnz != k.nnz || s.p != k.p || s.i != k.i)
    {
        g_plans.erase(it); // a different object now lives at this address
        return nullptr;
    }
    return dynamic_cast<PlanT *>(it->second.get());
}

void drop_plan(const void *obj)
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_plans.erase(obj);
}

void check_csr(const CSR_matrix *A, const char *what)
{
    if (!A) fail(SDL_ERR_INVALID, std::string(what) + " is NULL");
    if (A->m < 0 || A->n < 0 || A->nnz < 0) fail(SDL_ERR_INVALID, std::string(what) + ": negative size");
    if (!A->p || (A->nnz > 0 && !A->i)) fail(SDL_ERR_INVALID, std::string(what) + ": NULL arrays");
}
void check_csc(const CSC_matrix *A, const char *what)
{
    if (!A) fail(SDL_ERR_INVALID, std::string(what) + " is NULL");
    if (A->m < 0 || A->n < 0 || A->nnz < 0) fail(SDL_ERR_INVALID, std::string(what) + ": negative size");
    if (!A->p || (A->nnz > 0 && !A->i)) fail(SDL_ERR_INVALID, std::string(what) + ": NULL arrays");
}

// Builds the transpose plan of a compressed structure and returns it with the
// host copies of (Tp, Ti) written into out_p / out_i.
std::unique_ptr<TransposeRawPlan> build_transpose(const int *p, const int *idx, int rows, int cols,
                                                  int nnz, int *out_p, int *out_i)
{
    Runtime &rt = runtime();
    cudaStream_t s = rt.stream;
    auto plan = std::make_unique<TransposeRawPlan>();
    plan->rows = rows;
    plan->cols = cols;
    plan->nnz = nnz;
    DevBuf<int> dp = upload(p, (size_t)rows + 1, s), di = upload(idx, nnz, s);
    validate_compressed(dp.get(), di.get(), rows, cols, nnz, "transpose operand", s);
    transpose_build(dp.get(), di.get(), rows, cols, nnz, plan->T, s);
    d2h(out_p, plan->T.Tp.get(), (size_t)cols + 1, s);
    d2h(out_i, plan->T.Ti.get(), nnz, s);
    plan->x.reset(std::max(1, nnz));
    plan->Tx.reset(std::max(1, nnz));
    SDL_CUDA(cudaStreamSynchronize(s));
    return plan;
}

void run_transpose_fill(TransposeRawPlan *plan, const double *x, double *out)
{
    cudaStream_t s = runtime().stream;
    h2d(plan->x.get(), x, plan->nnz, s);
    gather_values(plan->T.src.get(), plan->x.get(), plan->Tx.get(), plan->nnz, s);
    d2h(out, plan->Tx.get(), plan->nnz, s);
    SDL_CUDA(cudaStreamSynchronize(s));
}

} // namespace

void raw_forget(const void *obj) { drop_plan(obj); }

// ------------------------------------------------------------------ pinning
namespace {
struct HostArr
{
    size_t bytes = 0;
    int state = 0; // 0 = pageable, 1 = registered, 2 = registration refused
};
std::mutex g_pin_mu;
std::unordered_map<const void *, HostArr> g_host;
constexpr size_t PIN_MIN_BYTES = 1u << 20;
} // namespace

void host_track(void *p, size_t bytes)
{
    if (!p || bytes < PIN_MIN_BYTES) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_host[p] = HostArr{bytes, 0};
}

void host_untrack(void *p)
{
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    auto it = g_host.find(p);
    if (it == g_host.end()) return;
    if (it->second.state == 1)
    {
        cudaHostUnregister(p);
        cudaGetLastError();
    }
    g_host.erase(it);
}

void host_pin_if_owned(const void *p, size_t bytes)
{
    if (bytes < PIN_MIN_BYTES) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    auto it = g_host.find(p);
    if (it == g_host.end() || it->second.state != 0) return;
    cudaError_t e = cudaHostRegister(const_cast<void *>(p), it->second.bytes, cudaHostRegisterDefault);
    if (e == cudaSuccess)
        it->second.state = 1;
    else
    {
        cudaGetLastError();
        it->second.state = 2;
    }
}

} // namespace sdl

using namespace sdl;

// ====================================================================== CSR
extern "C" CSR_matrix *new_CSR_matrix(int m, int n, int nnz)
{
    CSR_matrix *A = (CSR_matrix *)sp_malloc(sizeof(CSR_matrix));
    if (!A) return NULL;
    A->p = (int *)sp_calloc((size_t)m + 1, sizeof(int));
    A->i = (int *)sp_calloc(nnz > 0 ? (size_t)nnz : 1, sizeof(int));
    A->x = (double *)sp_malloc((nnz > 0 ? (size_t)nnz : 1) * sizeof(double));
    A->m = m;
    A->n = n;
    A->nnz = nnz;
    if (nnz > 0) host_track(A->x, (size_t)nnz * sizeof(double));
    return A;
}

extern "C" CSR_matrix *new_csr(const CSR_matrix *A)
{
    CSR_matrix *C = new_CSR_matrix(A->m, A->n, A->nnz);
    std::memcpy(C->p, A->p, ((size_t)A->m + 1) * sizeof(int));
    if (A->nnz > 0)
    {
        std::memcpy(C->i, A->i, (size_t)A->nnz * sizeof(int));
        std::memcpy(C->x, A->x, (size_t)A->nnz * sizeof(double));
    }
    return C;
}

extern "C" void free_CSR_matrix(CSR_matrix *matrix)
{
    if (!matrix) return;
    raw_forget(matrix);
    host_untrack(matrix->x);
    sp_free(matrix->p);
    sp_free(matrix->i);
    sp_free(matrix->x);
    sp_free(matrix);
}

extern "C" void copy_CSR_matrix(const CSR_matrix *A, CSR_matrix *C)
{
    C->m = A->m;
    C->n = A->n;
    C->nnz = A->nnz;
    std::memcpy(C->p, A->p, ((size_t)A->m + 1) * sizeof(int));
    if (A->nnz > 0)
    {
        std::memcpy(C->i, A->i, (size_t)A->nnz * sizeof(int));
        std::memcpy(C->x, A->x, (size_t)A->nnz * sizeof(double));
    }
}

extern "C" void CSR_trim(CSR_matrix *A)
{
    int nnz = A->p[A->m];
    A->nnz = nnz;
    if (nnz == 0) return;
    host_untrack(A->x);
    A->i = (int *)sp_realloc(A->i, (size_t)nnz * sizeof(int));
    A->x = (double *)sp_realloc(A->x, (size_t)nnz * sizeof(double));
    host_track(A->x, (size_t)nnz * sizeof(double));
}

extern "C" CSR_matrix *AT_alloc(const CSR_matrix *A, int *iwork)
{
    (void)iwork;
    return guard_upstream<CSR_matrix *>("AT_alloc", nullptr, [&]() -> CSR_matrix * {
        check_csr(A, "A");
        CSR_matrix *AT = new_CSR_matrix(A->n, A->m, A->nnz);
        try
        {
            auto plan = build_transpose(A->p, A->i, A->m, A->n, A->nnz, AT->p, AT->i);
            plan->key = key_of(AT);
            put_plan(std::move(plan));
        }
        catch (...)
        {
            free_CSR_matrix(AT);
            throw;
        }
        return AT;
    });
}

extern "C" void AT_fill_values(const CSR_matrix *A, CSR_matrix *AT, int *iwork)
{
    (void)iwork;
    guard_upstream_void("AT_fill_values", [&]() {
        check_csr(A, "A");
        auto *plan = find_plan<TransposeRawPlan>(AT);
        if (!plan)
        {
            // AT was not built by AT_alloc: build its plan now (one time).
            auto fresh = build_transpose(A->p, A->i, A->m, A->n, A->nnz, AT->p, AT->i);
            fresh->key = key_of(AT);
            plan = fresh.get();
            put_plan(std::move(fresh));
        }
        if (plan->rows != A->m || plan->cols != A->n || plan->nnz != A->nnz)
            fail(SDL_ERR_INVALID, "A does not match the structure AT was allocated for");
        run_transpose_fill(plan, A->x, AT->x);
    });
}

extern "C" CSR_matrix *transpose(const CSR_matrix *A, int *iwork)
{
    CSR_matrix *AT = AT_alloc(A, iwork);
    if (AT) AT_fill_values(A, AT, iwork);
    return AT;
}

// ====================================================================== CSC
extern "C" CSC_matrix *new_CSC_matrix(int m, int n, int nnz)
{
    CSC_matrix *A = (CSC_matrix *)sp_malloc(sizeof(CSC_matrix));
    if (!A) return NULL;
    A->p = (int *)sp_malloc(((size_t)n + 1) * sizeof(int));
    A->i = (int *)sp_malloc((nnz > 0 ? (size_t)nnz : 1) * sizeof(int));
    A->x = (double *)sp_malloc((nnz > 0 ? (size_t)nnz : 1) * sizeof(double));
    if (!A->p || !A->i || !A->x)
    {
        sp_free(A->p);
        sp_free(A->i);
        sp_free(A->x);
        sp_free(A);
        return NULL;
    }
    A->m = m;
    A->n = n;
    A->nnz = nnz;
    if (nnz > 0) host_track(A->x, (size_t)nnz * sizeof(double));
    return A;
}

extern "C" void free_CSC_matrix(CSC_matrix *matrix)
{
    if (!matrix) return;
    raw_forget(matrix);
    host_untrack(matrix->x);
    sp_free(matrix->p);
    sp_free(matrix->i);
    sp_free(matrix->x);
    sp_free(matrix);
}

extern "C" CSC_matrix *csr_to_csc_alloc(const CSR_matrix *A, int *iwork)
{
    (void)iwork;
    return guard_upstream<CSC_matrix *>("csr_to_csc_alloc", nullptr, [&]() -> CSC_matrix * {
        check_csr(A, "A");
        CSC_matrix *C = new_CSC_matrix(A->m, A->n, A->nnz);
        if (!C) throw std::bad_alloc();
        try
        {
            auto plan = build_transpose(A->p, A->i, A->m, A->n, A->nnz, C->p, C->i);
            plan->key = key_of(C);
            put_plan(std::move(plan));
        }
        catch (...)
        {
            free_CSC_matrix(C);
            throw;
        }
        return C;
    });
}

extern "C" void csr_to_csc_fill_values(const CSR_matrix *A, CSC_matrix *C, int *iwork)
{
    (void)iwork;
    guard_upstream_void("csr_to_csc_fill_values", [&]() {
        check_csr(A, "A");
        auto *plan = find_plan<TransposeRawPlan>(C);
        if (!plan)
        {
            auto fresh = build_transpose(A->p, A->i, A->m, A->n, A->nnz, C->p, C->i);
            fresh->key = key_of(C);
            plan = fresh.get();
            put_plan(std::move(fresh));
        }
        if (plan->rows != A->m || plan->cols != A->n || plan->nnz != A->nnz)
            fail(SDL_ERR_INVALID, "A does not match the structure C was allocated for");
        run_transpose_fill(plan, A->x, C->x);
    });
}

extern "C" CSR_matrix *csc_to_csr_alloc(const CSC_matrix *A, int *iwork)
{
    (void)iwork;
    return guard_upstream<CSR_matrix *>("csc_to_csr_alloc", nullptr, [&]() -> CSR_matrix * {
        check_csc(A, "A");
        CSR_matrix *C = new_CSR_matrix(A->m, A->n, A->nnz);
        try
        {
            // the columns of A are the rows of A^T: transposing them gives A's rows
            auto plan = build_transpose(A->p, A->i, A->n, A->m, A->nnz, C->p, C->i);
            plan->key = key_of(C);
            put_plan(std::move(plan));
        }
        catch (...)
        {
            free_CSR_matrix(C);
            throw;
        }
        return C;
    });
}

extern "C" void csc_to_csr_fill_values(const CSC_matrix *A, CSR_matrix *C, int *iwork)
{
    (void)iwork;
    guard_upstream_void("csc_to_csr_fill_values", [&]() {
        check_csc(A, "A");
        auto *plan = find_plan<TransposeRawPlan>(C);
        if (!plan)
        {
            auto fresh = build_transpose(A->p, A->i, A->n, A->m, A->nnz, C->p, C->i);
            fresh->key = key_of(C);
            plan = fresh.get();
            put_plan(std::move(fresh));
        }
        if (plan->rows != A->n || plan->cols != A->m || plan->nnz != A->nnz)
            fail(SDL_ERR_INVALID, "A does not match the structure C was allocated for");
        run_transpose_fill(plan, A->x, C->x);
    });
}

// ------------------------------------------------------------ B^T D A (raw)
namespace {
std::unique_ptr<ProductPlan> build_btda(const CSR_matrix *A, const CSC_matrix *B, CSR_matrix **outC)
{
    Runtime &rt = runtime();
    cudaStream_t s = rt.stream;
    if (A->m != B->m) fail(SDL_ERR_INVALID, "rows of A and B differ");
    auto plan = std::make_unique<ProductPlan>();
    plan->A_m = A->m;
    plan->A_n = A->n;
    plan->A_nnz = A->nnz;
    plan->B_m = B->m;
    plan->B_n = B->n;
    plan->B_nnz = B->nnz;
    plan->Ap = upload(A->p, (size_t)A->m + 1, s);
    plan->Ai = upload(A->i, A->nnz, s);
    plan->Lp = upload(B->p, (size_t)B->n + 1, s);
    plan->Li = upload(B->i, B->nnz, s);
    ProductDesc d;
    d.Lp = plan->Lp.get();
    d.Li = plan->Li.get();
    d.L_m = B->n;
    d.L_nnz = B->nnz;
    d.blocks = 1;
    d.Ap = plan->Ap.get();
    d.Ai = plan->Ai.get();
    d.A_m = A->m;
    d.A_n = A->n;
    d.A_nnz = A->nnz;
    product_symbolic(d, TuneConfig{}, plan->P, s);
    CSR_matrix *C = new_CSR_matrix(B->n, A->n, plan->P.nnz);
    d2h(C->p, plan->P.Cp.get(), (size_t)B->n + 1, s);
    d2h(C->i, plan->P.Ci.get(), plan->P.nnz, s);
    plan->Lx.reset(std::max(1, B->nnz));
    plan->Ax.reset(std::max(1, A->nnz));
    plan->dv.reset(std::max(1, A->m));
    plan->Cx.reset(std::max(1, plan->P.nnz));
    SDL_CUDA(cudaStreamSynchronize(s));
    *outC = C;
    return plan;
}
} // namespace

extern "C" CSR_matrix *BTA_alloc(const CSR_matrix *A, const CSC_matrix *B)
{
    return guard_upstream<CSR_matrix *>("BTA_alloc", nullptr, [&]() -> CSR_matrix * {
        check_csr(A, "A");
        check_csc(B, "B");
        CSR_matrix *C = nullptr;
        auto plan = build_btda(A, B, &C);
        plan->key = key_of(C);
        put_plan(std::move(plan));
        return C;
    });
}

extern "C" void BTDA_fill_values(const CSR_matrix *A, const CSC_matrix *B, const double *d,
                                 double *acc, CSR_matrix *C)
{
    (void)acc;
    guard_upstream_void("BTDA_fill_values", [&]() {
        check_csr(A, "A");
        check_csc(B, "B");
        check_csr(C, "C");
        auto *plan = find_plan<ProductPlan>(C);
        if (!plan)
        {
            // C did not come from BTA_alloc: compute its plan once and adopt C's
            // structure only if it is the exact product structure.
            CSR_matrix *tmp = nullptr;
            auto fresh = build_btda(A, B, &tmp);
            bool same = tmp->m == C->m && tmp->n == C->n && tmp->nnz == C->nnz &&
                        std::memcmp(tmp->p, C->p, ((size_t)C->m + 1) * sizeof(int)) == 0 &&
                        (C->nnz == 0 || std::memcmp(tmp->i, C->i, (size_t)C->nnz * sizeof(int)) == 0);
            free_CSR_matrix(tmp);
            if (!same) fail(SDL_ERR_INVALID, "C does not have the structure of B^T A");
            fresh->key = key_of(C);
            plan = fresh.get();
            put_plan(std::move(fresh));
        }
        if (plan->A_m != A->m || plan->A_n != A->n || plan->A_nnz != A->nnz ||
            plan->B_m != B->m || plan->B_n != B->n || plan->B_nnz != B->nnz)
            fail(SDL_ERR_INVALID, "A or B does not match the operands C was allocated for");
        cudaStream_t s = runtime().stream;
        h2d(plan->Ax.get(), A->x, A->nnz, s);
        h2d(plan->Lx.get(), B->x, B->nnz, s);
        if (d) h2d(plan->dv.get(), d, A->m, s);
        product_numeric(plan->P, plan->Lx.get(), d ? plan->dv.get() : nullptr, plan->Ax.get(),
                        plan->Cx.get(), s);
        d2h(C->x, plan->Cx.get(), plan->P.nnz, s);
        check_device_errors(s, "BTDA_fill_values");
    });
}

// ====================================================================== COO
extern "C" COO_matrix *new_COO_matrix(const CSR_matrix *A)
{
    COO_matrix *coo = (COO_matrix *)sp_malloc(sizeof(COO_matrix));
    size_t nz = A->nnz > 0 ? (size_t)A->nnz : 1;
    coo->m = A->m;
    coo->n = A->n;
    coo->nnz = A->nnz;
    coo->rows = (int *)sp_malloc(nz * sizeof(int));
    coo->cols = (int *)sp_malloc(nz * sizeof(int));
    coo->x = (double *)sp_malloc(nz * sizeof(double));
    coo->value_map = NULL;
    for (int r = 0; r < A->m; ++r)
        for (int k = A->p[r]; k < A->p[r + 1]; ++k) coo->rows[k] = r;
    if (A->nnz > 0)
    {
        std::memcpy(coo->cols, A->i, (size_t)A->nnz * sizeof(int));
        std::memcpy(coo->x, A->x, (size_t)A->nnz * sizeof(double));
    }
    return coo;
}

extern "C" COO_matrix *new_COO_matrix_lower_triangular(const CSR_matrix *A)
{
    int count = 0;
    for (int r = 0; r < A->m; ++r)
        for (int k = A->p[r]; k < A->p[r + 1]; ++k)
            if (A->i[k] <= r) ++count;
    COO_matrix *coo = (COO_matrix *)sp_malloc(sizeof(COO_matrix));
    size_t nz = count > 0 ? (size_t)count : 1;
    coo->m = A->m;
    coo->n = A->n;
    coo->nnz = count;
    coo->rows = (int *)sp_malloc(nz * sizeof(int));
    coo->cols = (int *)sp_malloc(nz * sizeof(int));
    coo->x = (double *)sp_malloc(nz * sizeof(double));
    coo->value_map = (int *)sp_malloc(nz * sizeof(int));
    int at = 0;
    for (int r = 0; r < A->m; ++r)
        for (int k = A->p[r]; k < A->p[r + 1]; ++k)
            if (A->i[k] <= r)
            {
                coo->rows[at] = r;
                coo->cols[at] = A->i[k];
                coo->x[at] = A->x[k];
                coo->value_map[at] = k;
                ++at;
            }
    return coo;
}

extern "C" void refresh_lower_triangular_coo(COO_matrix *coo, const double *vals)
{
    for (int k = 0; k < coo->nnz; ++k) coo->x[k] = vals[coo->value_map[k]];
}

extern "C" void free_COO_matrix(COO_matrix *matrix)
{
    if (!matrix) return;
    raw_forget(matrix);
    sp_free(matrix->rows);
    sp_free(matrix->cols);
    sp_free(matrix->x);
    sp_free(matrix->value_map);
    sp_free(matrix);
}

// ------------------------------------------------------------ COO coalesce
namespace {
std::unique_ptr<CoalesceRawPlan> build_coalesce(const COO_matrix *A, CSR_matrix **outC)
{
    cudaStream_t s = runtime().stream;
    auto plan = std::make_unique<CoalesceRawPlan>();
    plan->m = A->m;
    plan->n = A->n;
    plan->nnz_in = A->nnz;
    plan->rows = upload(A->rows, A->nnz, s);
    plan->cols = upload(A->cols, A->nnz, s);
    sdl_status st = sdl_coalesce_create(plan->rows.get(), plan->cols.get(), A->nnz, A->m, A->n, s,
                                        &plan->plan);
    if (st != SDL_OK) fail(st, sdl_last_error());
    int nnz = 0;
    const int *Cp = nullptr, *Ci = nullptr;
    sdl_coalesce_info(plan->plan, &nnz, &Cp, &Ci);
    CSR_matrix *C = new_CSR_matrix(A->m, A->n, nnz);
    d2h(C->p, Cp, (size_t)A->m + 1, s);
    d2h(C->i, Ci, nnz, s);
    plan->x.reset(std::max(1, A->nnz));
    plan->Cx.reset(std::max(1, nnz));
    SDL_CUDA(cudaStreamSynchronize(s));
    *outC = C;
    return plan;
}
} // namespace

extern "C" CSR_matrix *COO_coalesce_alloc(const COO_matrix *A)
{
    return guard_upstream<CSR_matrix *>("COO_coalesce_alloc", nullptr, [&]() -> CSR_matrix * {
        if (!A || A->m < 0 || A->n < 0 || A->nnz < 0) fail(SDL_ERR_INVALID, "bad COO matrix");
        CSR_matrix *C = nullptr;
        auto plan = build_coalesce(A, &C);
        plan->key = key_of(C);
        put_plan(std::move(plan));
        return C;
    });
}

extern "C" void COO_coalesce_fill_values(const COO_matrix *A, CSR_matrix *C)
{
    guard_upstream_void("COO_coalesce_fill_values", [&]() {
        if (!A || !C) fail(SDL_ERR_INVALID, "NULL argument");
        auto *plan = find_plan<CoalesceRawPlan>(C);
        if (!plan) fail(SDL_ERR_INVALID, "C was not built by COO_coalesce_alloc");
        if (plan->m != A->m || plan->n != A->n || plan->nnz_in != A->nnz)
            fail(SDL_ERR_INVALID, "A does not match the COO C was allocated for");
        cudaStream_t s = runtime().stream;
        h2d(plan->x.get(), A->x, A->nnz, s);
        sdl_status st = sdl_coalesce_fill(plan->plan, plan->x.get(), plan->Cx.get(), s);
        if (st != SDL_OK) fail(st, sdl_last_error());
        d2h(C->x, plan->Cx.get(), C->nnz, s);
        check_device_errors(s, "COO_coalesce_fill_values");
    });
}

// ====================================================================== status API
extern "C" sdl_status sdl_last_status(void) { return t_status; }
extern "C" const char *sdl_last_error(void) { return t_message.c_str(); }
extern "C" void sdl_clear_error(void)
{
    t_status = SDL_OK;
    t_message.clear();
}
extern "C" void sdl_set_fatal_errors(int fatal) { g_fatal.store(fatal ? 1 : 0); }
