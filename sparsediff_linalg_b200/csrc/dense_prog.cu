// Fill programs over dense blocks (declarations and the program model are in
// dense_prog.h). Every index a kernel reads is checked on the host when the
// program is built, against the sizes the fill accepts, so the kernels carry no
// per-access bounds checks of their own.
#include <algorithm>
#include <climits>
#include <map>

#include "dense_prog.h"
#include "sdl_device.cuh"

namespace sdl {
namespace {

int grid_cap3(long long work_items, int per_block, int cap)
{
    long long g = (work_items + per_block - 1) / per_block;
    return (int)std::max<long long>(1, std::min<long long>(g, cap));
}

__device__ __forceinline__ void mma_f64_acc(double &c0, double &c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// One warp per row task, lanes on the row's values.
__global__ void __launch_bounds__(256) k_dp_rows(const DpRowTask *__restrict__ tasks, int n,
                                                 const long long *__restrict__ src, const double *__restrict__ XL,
                                                 const double *__restrict__ d, double *__restrict__ P)
{
    const int w = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (w >= n) return;
    const int lane = threadIdx.x & 31;
    const DpRowTask T = tasks[w];
    double *dst = P + T.dst;
    if (T.mode == DP_ROW_SUM)
    {
        for (int j = lane; j < T.len; j += 32)
        {
            double acc = 0.0;
            for (int e = T.e_begin; e < T.e_end; ++e) acc = __dadd_rn(acc, XL[src[e] + j]);
            dst[j] = acc;
        }
        return;
    }
    const double *s = XL + src[T.e_begin];
    if (T.mode == DP_ROW_SCALE)
    {
        const double f = d[T.scale_row];
        for (int j = lane; j < T.len; j += 32) dst[j] = __dmul_rn(s[j], f);
    }
    else
        for (int j = lane; j < T.len; j += 32) dst[j] = s[j];
}

// 32 x 32 tiles through shared memory; 32 x 8 threads.
__global__ void __launch_bounds__(256) k_dp_transpose(const DpTrTask *__restrict__ tasks,
                                                      const int4 *__restrict__ tiles, int ntiles,
                                                      const double *__restrict__ XL, double *__restrict__ P)
{
    __shared__ double tile[32][33];
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    {
        const int4 tl = tiles[t];
        const DpTrTask T = tasks[tl.x];
        const int r0 = tl.y, c0 = tl.z;
        const double *A = XL + T.src;
        for (int y = threadIdx.y; y < 32; y += 8)
        {
            const int r = r0 + y, c = c0 + threadIdx.x;
            if (r < T.m0 && c < T.n0) tile[y][threadIdx.x] = A[(long long)r * T.n0 + c];
        }
        __syncthreads();
        double *C = P + T.dst; // n0 x m0
        for (int y = threadIdx.y; y < 32; y += 8)
        {
            const int c = c0 + y, r = r0 + threadIdx.x;
            if (c < T.n0 && r < T.m0) C[(long long)c * T.m0 + r] = tile[threadIdx.x][y];
        }
        __syncthreads();
    }
}

// One warp per 16 x 16 tile of a gathered GEMM: four m8n8k4 accumulators, K in
// ascending gathered-row order, four rows per step.
//   A fragment: lane holds L(a0 + 8h + lane / 4, t = k + lane % 4)
//   B fragment: lane holds R(t = k + lane % 4, b0 + 8h + lane / 4)
//   C: lane holds rows a0 + 8h + lane / 4, columns b0 + 8h' + 2 (lane % 4) + {0, 1}
__global__ void __launch_bounds__(128) k_dp_gemm(const DpGemmTask *__restrict__ tasks,
                                                 const int4 *__restrict__ tiles, int ntiles,
                                                 const int *__restrict__ lidx, const int *__restrict__ ridx,
                                                 const int *__restrict__ drow, const double *__restrict__ XL,
                                                 const double *__restrict__ XR, const double *__restrict__ d,
                                                 double *__restrict__ P)
{
    const int w = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (w >= ntiles) return;
    const int lane = threadIdx.x & 31;
    const int4 tl = tiles[w];
    const DpGemmTask T = tasks[tl.x];
    const int a0 = tl.y, b0 = tl.z;
    const int g = lane >> 2, q = lane & 3;
    const double *L = XL + T.l_off, *R = XR + T.r_off;
    double c[2][2][2] = {};
    for (int k = 0; k < T.s; k += 4)
    {
        const int t = k + q;
        const bool ok = t < T.s;
        const long long it = T.idx_off + (ok ? t : 0);
        const int li = ok ? lidx[it] : 0, ri = ok ? ridx[it] : 0;
        const double dv = (ok && d) ? d[drow[it]] : 1.0;
        double a[2], b[2];
#pragma unroll
        for (int h = 0; h < 2; ++h)
        {
            const int i = a0 + 8 * h + g, j = b0 + 8 * h + g;
            a[h] = (ok && i < T.ni)
                       ? L[T.l_trans ? (long long)li * T.l_ld + i : (long long)i * T.l_ld + li]
                       : 0.0;
            const double xr = (ok && j < T.nj) ? R[(long long)ri * T.r_ld + j] : 0.0;
            b[h] = d ? __dmul_rn(xr, dv) : xr;
        }
#pragma unroll
        for (int ha = 0; ha < 2; ++ha)
#pragma unroll
            for (int hb = 0; hb < 2; ++hb) mma_f64_acc(c[ha][hb][0], c[ha][hb][1], a[ha], b[hb]);
    }
    double *Pt = P + T.p;
#pragma unroll
    for (int ha = 0; ha < 2; ++ha)
#pragma unroll
        for (int hb = 0; hb < 2; ++hb)
#pragma unroll
            for (int e = 0; e < 2; ++e)
            {
                const int r = a0 + 8 * ha + g, cc = b0 + 8 * hb + 2 * q + e;
                if (r < T.ni && cc < T.nj) Pt[(long long)r * T.nj + cc] = c[ha][hb][e];
            }
}

// One warp per sparse x dense vector; lanes on the vector's values.
__global__ void __launch_bounds__(256) k_dp_spvec(const DpSpTask *__restrict__ tasks, int n,
                                                  const int *__restrict__ e_kk, const int *__restrict__ e_pos,
                                                  const int *__restrict__ e_row, const double *__restrict__ XL,
                                                  const double *__restrict__ XR, const double *__restrict__ Sx,
                                                  const double *__restrict__ d, double *__restrict__ P)
{
    const int w = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (w >= n) return;
    const int lane = threadIdx.x & 31;
    const DpSpTask T = tasks[w];
    const double *X = (T.dense_right ? XR : XL) + T.x_off;
    for (int t = lane; t < T.nvec; t += 32)
    {
        double acc = 0.0;
        for (int e = T.e_begin; e < T.e_end; ++e)
        {
            const double x = T.dense_trans ? X[(long long)t * T.ld + e_kk[e]] : X[(long long)e_kk[e] * T.ld + t];
            const double sv = Sx[e_pos[e]];
            double term;
            if (d && T.mode == DP_SP_D_DENSE)
                term = __dmul_rn(sv, __dmul_rn(d[e_row[e]], x));
            else if (d && T.mode == DP_SP_D_SPARSE)
                term = __dmul_rn(__dmul_rn(d[e_row[e]], sv), x);
            else
                term = __dmul_rn(sv, x);
            acc = __dadd_rn(acc, term);
        }
        P[T.p + (long long)t * T.stride] = acc;
    }
}

// Output cells of stage 2; grid.y = output blocks.
__global__ void k_dp_gather(const DpOut *__restrict__ outd, int o_base, const DpSrc *__restrict__ srcs,
                            const int *__restrict__ maps, const double *__restrict__ P, double *__restrict__ C)
{
    const DpOut D = outd[o_base + blockIdx.y];
    const long long cells = (long long)D.m0 * D.n0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < cells;
         e += (long long)gridDim.x * blockDim.x)
    {
        const int i = (int)(e / D.n0), j = (int)(e - (long long)i * D.n0);
        const int *mp = maps + D.map_off;
        double acc = 0.0;
        for (int t = D.s_begin; t < D.s_end; ++t, mp += D.m0 + D.n0)
        {
            const int si = mp[i], sj = mp[D.m0 + j];
            if (si < 0 || sj < 0) continue;
            const DpSrc S = srcs[t];
            const double v = P[S.p + (long long)si * S.rs + (long long)sj * S.cs];
            if (!D.accumulate)
            {
                acc = v;
                break;
            }
            acc = __dadd_rn(acc, v);
        }
        C[D.c_off + e] = acc;
    }
}

[[noreturn]] void bad_prog(const char *what) { fail(SDL_ERR_INTERNAL, std::string("dense-block program: ") + what); }

// Upload the stage-1 tasks and their tiles.
void dp_upload_stage1(DenseProg &P, DpBuilder &b, cudaStream_t s)
{
    P.n_row = (int)b.row.size();
    P.row = upload(b.row.data(), b.row.size(), s);
    P.row_src = upload(b.row_src.data(), b.row_src.size(), s);
    P.tr = upload(b.tr.data(), b.tr.size(), s);
    std::vector<int4> trt;
    for (size_t k = 0; k < b.tr.size(); ++k)
        for (int r = 0; r < b.tr[k].m0; r += 32)
            for (int c = 0; c < b.tr[k].n0; c += 32) trt.push_back(make_int4((int)k, r, c, 0));
    P.n_trt = (int)trt.size();
    P.tr_tiles = upload(trt.data(), trt.size(), s);
    P.gm = upload(b.gm.data(), b.gm.size(), s);
    std::vector<int4> gmt;
    for (size_t k = 0; k < b.gm.size(); ++k)
        for (int a = 0; a < b.gm[k].ni; a += 16)
            for (int c = 0; c < b.gm[k].nj; c += 16) gmt.push_back(make_int4((int)k, a, c, 0));
    P.n_gmt = (int)gmt.size();
    P.gm_tiles = upload(gmt.data(), gmt.size(), s);
    P.lidx = upload(b.lidx.data(), b.lidx.size(), s);
    P.ridx = upload(b.ridx.data(), b.ridx.size(), s);
    P.drow = upload(b.drow.data(), b.drow.size(), s);
    P.n_sp = (int)b.sp.size();
    P.sp = upload(b.sp.data(), b.sp.size(), s);
    P.e_kk = upload(b.e_kk.data(), b.e_kk.size(), s);
    P.e_pos = upload(b.e_pos.data(), b.e_pos.size(), s);
    P.e_row = upload(b.e_row.data(), b.e_row.size(), s);
    P.p_total = b.p_total;
}

} // namespace

void DpBuilder::row_copy(long long dst, long long src, int len, int mode, int scale_row)
{
    if (len <= 0) return;
    row.push_back(DpRowTask{dst, len, (int)row_src.size(), (int)row_src.size() + 1, scale_row, mode});
    row_src.push_back(src);
}

void DpBuilder::row_sum(long long dst, const std::vector<long long> &srcs, int len)
{
    if (len <= 0) return;
    if ((long long)row_src.size() + (long long)srcs.size() > INT_MAX) fail(SDL_ERR_OVERFLOW, "dense-block program too large");
    row.push_back(DpRowTask{dst, len, (int)row_src.size(), (int)(row_src.size() + srcs.size()), -1, DP_ROW_SUM});
    row_src.insert(row_src.end(), srcs.begin(), srcs.end());
}

void DpBuilder::transpose(long long src, long long dst, int m0, int n0)
{
    if (m0 <= 0 || n0 <= 0) return;
    tr.push_back(DpTrTask{src, dst, m0, n0});
}

void DpBuilder::gemm(long long p, int ni, int nj, long long l_off, int l_ld, bool l_trans, const std::vector<int> &li,
                     long long r_off, int r_ld, const std::vector<int> &ri, const std::vector<int> &dr)
{
    if (ni <= 0 || nj <= 0) return;
    const long long off = (long long)lidx.size();
    gm.push_back(DpGemmTask{l_off, r_off, p, off, l_ld, r_ld, ni, nj, (int)li.size(), l_trans ? 1 : 0});
    lidx.insert(lidx.end(), li.begin(), li.end());
    ridx.insert(ridx.end(), ri.begin(), ri.end());
    drow.insert(drow.end(), dr.begin(), dr.end());
}

void DpBuilder::spvec(long long p, int nvec, int stride, long long x_off, int ld, bool dense_right, int mode,
                      const std::vector<int> &kk, const std::vector<int> &pos, const std::vector<int> &grow,
                      bool dense_trans)
{
    if (nvec <= 0) return;
    if ((long long)e_kk.size() + (long long)kk.size() > INT_MAX) fail(SDL_ERR_OVERFLOW, "dense-block program too large");
    sp.push_back(DpSpTask{x_off, p, ld, nvec, (int)e_kk.size(), (int)(e_kk.size() + kk.size()), stride, mode,
                          dense_right ? 1 : 0, dense_trans ? 1 : 0});
    e_kk.insert(e_kk.end(), kk.begin(), kk.end());
    e_pos.insert(e_pos.end(), pos.begin(), pos.end());
    e_row.insert(e_row.end(), grow.begin(), grow.end());
}

// Host check of every index the stage-1 kernels will read or write.
static void dp_validate(const DpBuilder &b, long long nl, long long nr, int ns, int d_len)
{
    const long long pt = b.p_total;
    for (const DpRowTask &t : b.row)
    {
        if (t.dst < 0 || t.dst + t.len > pt) bad_prog("row task writes outside the partials");
        for (int e = t.e_begin; e < t.e_end; ++e)
            if (b.row_src[e] < 0 || b.row_src[e] + t.len > nl) bad_prog("row task reads outside the operand");
        if (t.mode == DP_ROW_SCALE && (t.scale_row < 0 || t.scale_row >= d_len)) bad_prog("row scale outside d");
        if (t.mode != DP_ROW_SUM && t.e_end != t.e_begin + 1) bad_prog("row copy needs one source");
    }
    for (const DpTrTask &t : b.tr)
        if (t.src < 0 || t.dst < 0 || t.src + (long long)t.m0 * t.n0 > nl || t.dst + (long long)t.m0 * t.n0 > pt)
            bad_prog("transpose outside its buffers");
    for (const DpGemmTask &t : b.gm)
    {
        if (t.p < 0 || t.p + (long long)t.ni * t.nj > pt) bad_prog("GEMM writes outside the partials");
        for (int q = 0; q < t.s; ++q)
        {
            const long long li = b.lidx[t.idx_off + q], ri = b.ridx[t.idx_off + q];
            const long long lmax = t.l_trans ? li * t.l_ld + (t.ni - 1) : (long long)(t.ni - 1) * t.l_ld + li;
            if (li < 0 || t.l_off < 0 || t.l_off + lmax >= nl) bad_prog("GEMM reads outside the left operand");
            if (ri < 0 || t.r_off < 0 || t.r_off + ri * t.r_ld + (t.nj - 1) >= nr)
                bad_prog("GEMM reads outside the right operand");
            if (d_len > 0 && (b.drow[t.idx_off + q] < 0 || b.drow[t.idx_off + q] >= d_len))
                bad_prog("GEMM row outside d");
        }
    }
    for (const DpSpTask &t : b.sp)
    {
        if (t.p < 0 || t.p + (long long)(t.nvec - 1) * t.stride >= pt) bad_prog("vector writes outside the partials");
        const long long nx = t.dense_right ? nr : nl;
        for (int e = t.e_begin; e < t.e_end; ++e)
        {
            const long long last = t.dense_trans ? (long long)(t.nvec - 1) * t.ld + b.e_kk[e]
                                                 : (long long)b.e_kk[e] * t.ld + (t.nvec - 1);
            if (b.e_kk[e] < 0 || t.x_off < 0 || t.x_off + last >= nx) bad_prog("vector reads outside the dense operand");
            if (b.e_pos[e] < 0 || b.e_pos[e] >= ns) bad_prog("vector reads outside the sparse values");
            if (d_len > 0 && (b.e_row[e] < 0 || b.e_row[e] >= d_len)) bad_prog("vector row outside d");
        }
    }
}

std::unique_ptr<DenseProg> dp_direct(DpBuilder &b, long long c_total, cudaStream_t s)
{
    (void)s;
    auto P = std::make_unique<DenseProg>();
    if (b.p_total != c_total) bad_prog("direct program does not cover the output");
    P->c_total = c_total;
    return P;
}

namespace {

// Stage 2 from the output blocks (rows, cols) and, per output block, its value
// sources (partial index into `parts`, value index).
void dp_stage2(DenseProg &P, const DpBuilder &b, const std::vector<DpPart> &parts, const std::vector<int> &order,
               bool accumulate, cudaStream_t s)
{
    std::vector<DpOut> od;
    std::vector<DpSrc> hs;
    std::vector<int> hm;
    int nrows = 0, ncols = 0;
    for (const auto &r : P.out_rows)
        if (!r.empty()) nrows = std::max(nrows, r.back() + 1);
    for (const auto &c : P.out_cols)
        if (!c.empty()) ncols = std::max(ncols, c.back() + 1);
    for (const DpPart &pt : parts)
    {
        if (!pt.rows.empty()) nrows = std::max(nrows, pt.rows.back() + 1);
        if (!pt.cols.empty()) ncols = std::max(ncols, pt.cols.back() + 1);
    }
    std::vector<int> rpos(std::max(1, nrows), -1), cpos(std::max(1, ncols), -1);
    long long c_off = 0;
    P.max_cells = 0;
    for (int o = 0; o < P.n_out; ++o)
    {
        const std::vector<int> &rows = P.out_rows[o], &cols = P.out_cols[o];
        DpOut D{};
        D.c_off = c_off;
        D.m0 = (int)rows.size();
        D.n0 = (int)cols.size();
        if ((long long)D.m0 * D.n0 > INT_MAX) fail(SDL_ERR_OVERFLOW, "dense blocks: output block exceeds INT_MAX values");
        D.accumulate = accumulate ? 1 : 0;
        D.s_begin = (int)hs.size();
        D.map_off = (long long)hm.size();
        for (int k : P.out_srcs[o])
        {
            const DpPart &pt = parts[order.empty() ? k : order[k]];
            for (size_t q = 0; q < pt.rows.size(); ++q) rpos[pt.rows[q]] = (int)q;
            for (const DpPart::Val &v : pt.vals)
            {
                for (size_t q = 0; q < v.cols.size(); ++q) cpos[v.cols[q]] = (int)q;
                hs.push_back(DpSrc{v.p, v.rs, v.cs});
                const long long last = v.p + (long long)(pt.rows.size() ? pt.rows.size() - 1 : 0) * v.rs +
                                       (long long)(v.cols.size() ? v.cols.size() - 1 : 0) * v.cs;
                if (!pt.rows.empty() && !v.cols.empty() && (v.p < 0 || last >= b.p_total))
                    bad_prog("gather source outside the partials");
                for (int r : rows) hm.push_back(rpos[r]);
                for (int c : cols) hm.push_back(cpos[c]);
                for (int c : v.cols) cpos[c] = -1;
            }
            for (int r : pt.rows) rpos[r] = -1;
        }
        D.s_end = (int)hs.size();
        od.push_back(D);
        c_off += (long long)D.m0 * D.n0;
        P.max_cells = std::max(P.max_cells, (long long)D.m0 * D.n0);
    }
    P.c_total = c_off;
    P.outd = upload(od.data(), od.size(), s);
    P.srcs = upload(hs.data(), hs.size(), s);
    P.maps = upload(hm.data(), hm.size(), s);
    P.P.reset((size_t)std::max<long long>(1, b.p_total));
    P.gathered = true;
}

} // namespace

std::unique_ptr<DenseProg> dp_coalesced(DpBuilder &b, const std::vector<DpPart> &parts, int nrows, int ncols,
                                        bool accumulate, cudaStream_t s)
{
    auto P = std::make_unique<DenseProg>();
    const int n_src = (int)parts.size();
    std::vector<std::vector<int>> row_parts(std::max(1, nrows));
    for (int k = 0; k < n_src; ++k)
        for (int r : parts[k].rows)
        {
            if (r < 0 || r >= nrows) bad_prog("partial row outside the result");
            row_parts[r].push_back(k);
        }
    for (const DpPart &pt : parts)
        for (int c : pt.cols)
            if (c < 0 || c >= ncols) bad_prog("partial column outside the result");
    std::map<std::vector<int>, int> sig_id;
    for (int r = 0; r < nrows; ++r)
    {
        if (row_parts[r].empty()) continue;
        auto it = sig_id.find(row_parts[r]);
        int sid;
        if (it == sig_id.end())
        {
            sid = (int)P->out_rows.size();
            sig_id.emplace(row_parts[r], sid);
            P->out_rows.emplace_back();
            P->out_srcs.push_back(row_parts[r]);
        }
        else
            sid = it->second;
        P->out_rows[sid].push_back(r);
    }
    P->n_out = (int)P->out_rows.size();
    for (int o = 0; o < P->n_out; ++o)
    {
        std::vector<int> cols;
        for (int k : P->out_srcs[o]) cols.insert(cols.end(), parts[k].cols.begin(), parts[k].cols.end());
        std::sort(cols.begin(), cols.end());
        cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
        P->out_cols.push_back(std::move(cols));
    }
    dp_stage2(*P, b, parts, {}, accumulate, s);
    return P;
}

std::unique_ptr<DenseProg> dp_blocks(DpBuilder &b, const std::vector<DpPart> &parts, cudaStream_t s)
{
    auto P = std::make_unique<DenseProg>();
    P->n_out = (int)parts.size();
    for (size_t k = 0; k < parts.size(); ++k)
    {
        P->out_rows.push_back(parts[k].rows);
        P->out_cols.push_back(parts[k].cols);
        P->out_srcs.push_back({(int)k});
    }
    dp_stage2(*P, b, parts, {}, true, s);
    return P;
}

std::unique_ptr<DenseProg> dp_single(DpBuilder &b, const std::vector<int> &rows, const std::vector<int> &cols,
                                     const std::vector<DpPart> &parts, cudaStream_t s)
{
    auto P = std::make_unique<DenseProg>();
    P->n_out = 1;
    P->out_rows = {rows};
    P->out_cols = {cols};
    std::vector<int> all(parts.size());
    for (size_t k = 0; k < parts.size(); ++k) all[k] = (int)k;
    P->out_srcs = {all};
    dp_stage2(*P, b, parts, {}, true, s);
    return P;
}

void dp_finish(DenseProg &P, DpBuilder &b, long long nl, long long nr, int ns, int d_len, cudaStream_t s)
{
    dp_validate(b, nl, nr, ns, d_len);
    P.nl = nl;
    P.nr = nr;
    P.ns = ns;
    P.d_len = d_len;
    for (const DpRowTask &t : b.row) P.needs_d |= t.mode == DP_ROW_SCALE;
    dp_upload_stage1(P, b, s);
    SDL_CUDA(cudaStreamSynchronize(s));
}

void dp_fill(DenseProg &P, const double *XL, const double *XR, const double *Sx, const double *d, double *C,
             cudaStream_t s)
{
    if (d && P.d_len <= 0) bad_prog("d given to a product without a diagonal");
    if (!d && P.needs_d) bad_prog("d missing");
    if (P.c_total == 0) return;
    double *dst = P.gathered ? P.P.get() : C;
    if (P.n_row > 0)
        SDL_LAUNCH(k_dp_rows, (P.n_row + 7) / 8, 256, 0, s, P.row.get(), P.n_row, P.row_src.get(), XL, d, dst);
    if (P.n_trt > 0)
        SDL_LAUNCH(k_dp_transpose, grid_cap3(P.n_trt, 1, 148 * 8), dim3(32, 8), 0, s, P.tr.get(), P.tr_tiles.get(),
                   P.n_trt, XL, dst);
    if (P.n_gmt > 0)
        SDL_LAUNCH(k_dp_gemm, (P.n_gmt + 3) / 4, 128, 0, s, P.gm.get(), P.gm_tiles.get(), P.n_gmt, P.lidx.get(),
                   P.ridx.get(), P.drow.get(), XL, XR, d, dst);
    if (P.n_sp > 0)
        SDL_LAUNCH(k_dp_spvec, (P.n_sp + 7) / 8, 256, 0, s, P.sp.get(), P.n_sp, P.e_kk.get(), P.e_pos.get(),
                   P.e_row.get(), XL, XR, Sx, d, dst);
    if (!P.gathered) return;
    for (int o = 0; o < P.n_out; o += 65535)
    {
        const dim3 grid(grid_cap3(P.max_cells, 256, 4096), (unsigned)std::min(65535, P.n_out - o));
        SDL_LAUNCH(k_dp_gather, grid, 256, 0, s, P.outd.get(), o, P.srcs.get(), P.maps.get(), P.P.get(), C);
    }
}

} // namespace sdl
