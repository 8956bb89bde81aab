// extern "C" entry points of libculipx (declared in include/culipx.h).
#include "factor.h"
#include "kkt_assembly.h"
#include "ldu.h"
#include "operators.h"
#include "pattern.h"
#include "permute.h"
#include "server.h"
#include "spmv.h"
#include "sqmr.h"

#include <cstring>
#include <new>
#include <vector>

namespace culipx {
const char* last_error();
}

using namespace culipx;

#define GUARD_BEGIN try {
#define GUARD_END                                                                            \
    }                                                                                        \
    catch (const std::bad_alloc&) { return fail(CULIPX_OOM, "host allocation failed"); }     \
    catch (...) { return fail(CULIPX_CUDA_ERROR, "unexpected exception"); }

namespace culipx {

void handle_retain(culipx_handle_t* h)
{
    if (h) h->refs.fetch_add(1, std::memory_order_relaxed);
}

void handle_release(culipx_handle_t* h)
{
    if (!h || h->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) return;
    if (h->device >= 0 && cudaSetDevice(h->device) != cudaSuccess) cudaGetLastError();
    delete h->sqmr;
    if (h->vec_scratch) cudaFree(h->vec_scratch);
    if (h->ev_start) cudaEventDestroy(h->ev_start);
    if (h->ev_stop) cudaEventDestroy(h->ev_stop);
    delete h;
}

}  // namespace culipx

namespace {

// references on a pattern (Pattern::refs); the last release frees it and
// drops its reference on the handle
void pattern_retain(Pattern* p) { p->refs.fetch_add(1, std::memory_order_relaxed); }

void pattern_release(Pattern* p)
{
    if (!p || p->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) return;
    culipx_handle_t* h = p->handle;
    if (h && h->device >= 0 && cudaSetDevice(h->device) != cudaSuccess) cudaGetLastError();
    delete static_cast<culipx_pattern_t*>(p);
    handle_release(h);
}

// makes the object's device current before it frees device memory
void set_device_of(const culipx_handle_t* h)
{
    if (h && h->device >= 0 && cudaSetDevice(h->device) != cudaSuccess) cudaGetLastError();
}

int use_device(culipx_handle_t* h)
{
    if (h->device < 0) return CULIPX_OK;  // host-only handle
    CULIPX_CUDA(cudaSetDevice(h->device));
    return CULIPX_OK;
}
}  // namespace

extern "C" {

CULIPX_API const char* culipx_last_error(void) { return last_error(); }

CULIPX_API int culipx_version(void) { return 10000; }

CULIPX_API int culipx_handle_create(culipx_handle* out, int device, void* cuda_stream)
{
    if (!out) return fail(CULIPX_INVALID_ARG, "culipx_handle_create: null out");
    GUARD_BEGIN
    if (device == -1) {
        // host-only handle: symbolic analysis without a device mirror
        auto* h = new culipx_handle_t();
        h->device = -1;
        h->sqmr = new Sqmr();
        *out = h;
        return CULIPX_OK;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(CULIPX_CUDA_ERROR, "culipx_handle_create: no CUDA device");
    }
    if (device < 0 || device >= ndev) return fail(CULIPX_INVALID_ARG, "culipx_handle_create: bad device %d", device);
    auto* h = new culipx_handle_t();
    h->device = device;
    h->stream = static_cast<cudaStream_t>(cuda_stream);
    if (cudaSetDevice(device) != cudaSuccess || cudaEventCreate(&h->ev_start) != cudaSuccess ||
        cudaEventCreate(&h->ev_stop) != cudaSuccess) {
        delete h;
        return fail(CULIPX_CUDA_ERROR, "culipx_handle_create: CUDA initialization failed");
    }
    h->sqmr = new Sqmr();
    *out = h;
    return CULIPX_OK;
    GUARD_END
}

CULIPX_API int culipx_handle_destroy(culipx_handle h)
{
    // objects created on the handle keep it alive until they are destroyed
    handle_release(h);
    return CULIPX_OK;
}

CULIPX_API int culipx_handle_set_stream(culipx_handle h, void* cuda_stream)
{
    if (!h) return fail(CULIPX_INVALID_ARG, "null handle");
    h->stream = static_cast<cudaStream_t>(cuda_stream);
    return CULIPX_OK;
}

CULIPX_API int culipx_handle_set_memory_budget(culipx_handle h, long long bytes)
{
    if (!h) return fail(CULIPX_INVALID_ARG, "null handle");
    h->budget = bytes;
    return CULIPX_OK;
}

CULIPX_API int culipx_handle_memory_used(culipx_handle h, long long* bytes)
{
    if (!h || !bytes) return fail(CULIPX_INVALID_ARG, "null argument");
    *bytes = h->used.load();
    return CULIPX_OK;
}

CULIPX_API int culipx_handle_launch_count(culipx_handle h, long long* count, int reset)
{
    if (!h || !count) return fail(CULIPX_INVALID_ARG, "null argument");
    *count = h->launches;
    if (reset) h->launches = 0;
    return CULIPX_OK;
}

CULIPX_API int culipx_handle_synchronize(culipx_handle h)
{
    if (!h) return fail(CULIPX_INVALID_ARG, "null handle");
    CULIPX_TRY(use_device(h));
    CULIPX_CUDA(cudaStreamSynchronize(h->stream));
    return CULIPX_OK;
}

CULIPX_API int culipx_pattern_analyze(culipx_handle h, int n, const int* h_rowptr, const int* h_colidx,
                                      int num_blocks, const int* h_block_starts, int fill_level,
                                      double fill_factor, int precision, culipx_pattern* out)
{
    if (!h) return fail(CULIPX_INVALID_ARG, "null handle");
    GUARD_BEGIN
    CULIPX_TRY(use_device(h));
    Pattern* p = nullptr;
    CULIPX_TRY(analyze_pattern(h, n, h_rowptr, h_colidx, num_blocks, h_block_starts, fill_level, fill_factor,
                               precision, &p));
    handle_retain(h);
    *out = static_cast<culipx_pattern>(p);
    return CULIPX_OK;
    GUARD_END
}

CULIPX_API int culipx_pattern_analyze_systems(culipx_handle h, int n, const int* h_rowptr, const int* h_colidx,
                                              int num_blocks, const int* h_block_starts, int fill_level,
                                              double fill_factor, int precision, int num_systems,
                                              const int* h_row_offsets, culipx_pattern* out)
{
    if (!h) return fail(CULIPX_INVALID_ARG, "null handle");
    if (num_systems < 1 || !h_row_offsets) return fail(CULIPX_INVALID_ARG, "culipx_pattern_analyze_systems: bad systems");
    GUARD_BEGIN
    CULIPX_TRY(use_device(h));
    Pattern* p = nullptr;
    CULIPX_TRY(analyze_pattern(h, n, h_rowptr, h_colidx, num_blocks, h_block_starts, fill_level, fill_factor,
                               precision, &p, num_systems, h_row_offsets));
    handle_retain(h);
    *out = static_cast<culipx_pattern>(p);
    return CULIPX_OK;
    GUARD_END
}

CULIPX_API int culipx_pattern_destroy(culipx_pattern p)
{
    // factors and batches made from the pattern keep it alive until they are destroyed
    pattern_release(p);
    return CULIPX_OK;
}

CULIPX_API int culipx_pattern_info(culipx_pattern p, long long* info)
{
    if (!p || !info) return fail(CULIPX_INVALID_ARG, "null argument");
    const long long v[16] = {p->n,          p->nnz,           p->num_blocks,     p->coarse_nnz,
                             p->fill_nnz,   p->num_levels,    p->num_sparse,     p->num_dense,
                             p->val_slots,  p->val_slots,     p->max_level_blocks, p->max_level_rows,
                             p->device_bytes, p->precision,   0,                 0};
    std::memcpy(info, v, sizeof(v));
    return CULIPX_OK;
}

CULIPX_API int culipx_pattern_export(culipx_pattern p, int* coarse_off, int* coarse_col, int* blk_nnzA,
                                     int* lvl_off, int* lvl_rows, int* lb_off, int* lb, int* sb_off, int* sb,
                                     int* fmt, int* max_nnz)
{
    if (!p) return fail(CULIPX_INVALID_ARG, "null pattern");
    auto cp = [](int* dst, const std::vector<int>& src) {
        if (dst && !src.empty()) std::memcpy(dst, src.data(), src.size() * sizeof(int));
    };
    cp(coarse_off, p->cs_off);
    cp(coarse_col, p->cs_col);
    cp(blk_nnzA, p->blk_nnzA);
    cp(lvl_off, p->lvl_off);
    cp(lvl_rows, p->lvl_rows);
    cp(lb_off, p->lb_off);
    cp(lb, p->lb);
    cp(sb_off, p->sb_off);
    cp(sb, p->sb);
    cp(fmt, p->fmt);
    cp(max_nnz, p->max_nnz);
    return CULIPX_OK;
}

CULIPX_API int culipx_factor_create(culipx_pattern p, culipx_factor* out)
{
    if (!p || !out) return fail(CULIPX_INVALID_ARG, "null argument");
    if (p->handle->device < 0) return fail(CULIPX_INVALID_ARG, "culipx_factor_create: pattern was analyzed on a host-only handle");
    GUARD_BEGIN
    CULIPX_TRY(use_device(p->handle));
    Factor* f = nullptr;
    CULIPX_TRY(factor_create(p, &f));
    pattern_retain(p);
    *out = static_cast<culipx_factor>(f);
    return CULIPX_OK;
    GUARD_END
}

CULIPX_API int culipx_factor_destroy(culipx_factor f)
{
    if (f) {
        Pattern* p = f->pat;
        set_device_of(p->handle);
        delete f;
        pattern_release(p);
    }
    return CULIPX_OK;
}

CULIPX_API int culipx_factor_compute(culipx_factor f, const void* d_vals, const int* h_is_piv, int pivot,
                                     double threshold)
{
    if (!f) return fail(CULIPX_INVALID_ARG, "null factor");
    GUARD_BEGIN
    CULIPX_TRY(use_device(f->pat->handle));
    return factor_compute(f, d_vals, h_is_piv, pivot, threshold);
    GUARD_END
}

CULIPX_API int culipx_factor_compute_graph(culipx_factor f, const void* d_vals, int pivot, double threshold)
{
    if (!f) return fail(CULIPX_INVALID_ARG, "null factor");
    GUARD_BEGIN
    CULIPX_TRY(use_device(f->pat->handle));
    return factor_compute_graph(f, d_vals, pivot, threshold);
    GUARD_END
}

CULIPX_API int culipx_factor_compute_host(culipx_factor f, const double* h_vals, const int* h_is_piv, int pivot,
                                          double threshold)
{
    if (!f || !h_vals) return fail(CULIPX_INVALID_ARG, "null argument");
    GUARD_BEGIN
    culipx_handle_t* h = f->pat->handle;
    CULIPX_TRY(use_device(h));
    const long long nnz = f->pat->nnz;
    DeviceBuffer tmp;
    if (f->precision == CULIPX_F64) {
        CULIPX_TRY(tmp.upload(h, h_vals, nnz * sizeof(double)));
    } else {
        std::vector<float> fv(h_vals, h_vals + nnz);
        CULIPX_TRY(tmp.upload(h, fv.data(), nnz * sizeof(float)));
    }
    return factor_compute(f, tmp.get(), h_is_piv, pivot, threshold);
    GUARD_END
}

CULIPX_API int culipx_factor_export_size(culipx_factor f, long long* entries)
{
    if (!f || !entries) return fail(CULIPX_INVALID_ARG, "null argument");
    GUARD_BEGIN
    CULIPX_TRY(use_device(f->pat->handle));
    return factor_export(f, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, entries);
    GUARD_END
}

CULIPX_API int culipx_factor_export(culipx_factor f, int* h_blk_nnz, long long* h_blk_off, int* h_idx, void* h_val,
                                    void* h_tri, int* h_is_piv, int* h_perm, int* h_got_extra)
{
    if (!f) return fail(CULIPX_INVALID_ARG, "null factor");
    GUARD_BEGIN
    CULIPX_TRY(use_device(f->pat->handle));
    return factor_export(f, h_blk_nnz, h_blk_off, h_idx, h_val, h_tri, h_is_piv, h_perm, h_got_extra, nullptr);
    GUARD_END
}

CULIPX_API int culipx_factor_stats(culipx_factor f, double* ms, int* launches)
{
    if (!f) return fail(CULIPX_INVALID_ARG, "null factor");
    if (!f->computed) return fail(CULIPX_INVALID_ARG, "culipx_factor_stats: factor not computed");
    culipx_handle_t* h = f->pat->handle;
    CULIPX_TRY(use_device(h));
    // the last factorization's device time (its events bracket the launches)
    CULIPX_CUDA(cudaEventSynchronize(h->ev_stop));
    CULIPX_CUDA(cudaEventElapsedTime(&f->last_ms, h->ev_start, h->ev_stop));
    if (ms) *ms = f->last_ms;
    if (launches) *launches = f->last_launches;
    return CULIPX_OK;
}

CULIPX_API int culipx_factor_info(culipx_factor f, long long* info8)
{
    if (!f || !info8) return fail(CULIPX_INVALID_ARG, "null argument");
    if (!f->computed) return fail(CULIPX_INVALID_ARG, "culipx_factor_info: factor not computed");
    GUARD_BEGIN
    culipx_handle_t* h = f->pat->handle;
    CULIPX_TRY(use_device(h));
    const Pattern& p = *f->pat;
    const int n = p.n, cm = p.num_blocks;
    int u_nnz = 0, simple = 0;
    std::vector<int> flags(cm);
    CULIPX_CUDA(cudaStreamSynchronize(h->stream));
    CULIPX_CUDA(cudaMemcpy(&u_nnz, f->u_off.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost));
    CULIPX_CUDA(cudaMemcpy(&simple, f->scan_s.as<int>() + cm, sizeof(int), cudaMemcpyDeviceToHost));
    if (cm) CULIPX_CUDA(cudaMemcpy(flags.data(), f->rowflags.get(), cm * sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<int> extra(p.coarse_nnz);
    if (p.coarse_nnz)
        CULIPX_CUDA(cudaMemcpy(extra.data(), f->got_extra.get(), p.coarse_nnz * sizeof(int), cudaMemcpyDeviceToHost));
    long long granted = 0;
    for (int v : extra) granted += (v > 0);
    long long tiles = 0, tile_slots = 0, two = 0;
    for (int I = 0; I < cm; ++I) {
        const long long hI = p.bs[I + 1] - p.bs[I];
        if (!(flags[I] & kRowIdentity)) {
            ++tiles;
            tile_slots += hI * (hI + 1) / 2;
        }
        if (flags[I] & kRowHas2x2) ++two;
    }
    info8[0] = u_nnz;       // stored strictly off-diagonal entries of U (= of U')
    info8[1] = tiles;       // block rows whose pivot tile is not the identity
    info8[2] = tile_slots;  // upper-triangle entries of those tiles
    info8[3] = simple;      // fine rows in simple block rows
    info8[4] = two;         // block rows with a 2x2 pivot
    info8[5] = f->vbytes;
    info8[6] = granted;     // blocks that drew extra capacity from the dropping pass's leftover pool
    info8[7] = 0;
    return CULIPX_OK;
    GUARD_END
}

CULIPX_API int culipx_factor_set_solve_algorithm(culipx_factor f, int algorithm, int sweeps)
{
    if (!f) return fail(CULIPX_INVALID_ARG, "null factor");
    if (algorithm < CULIPX_SOLVE_STRIPE || algorithm > CULIPX_SOLVE_JACOBI)
        return fail(CULIPX_INVALID_ARG, "culipx_factor_set_solve_algorithm: bad algorithm %d", algorithm);
    if (sweeps < 0) return fail(CULIPX_INVALID_ARG, "culipx_factor_set_solve_algorithm: sweeps < 0");
    f->solve_algorithm = algorithm;
    f->jacobi_sweeps = sweeps;
    return CULIPX_OK;
}

CULIPX_API int culipx_factor_set_pivot_fp64(culipx_factor f, double bound)
{
    if (!f) return fail(CULIPX_INVALID_ARG, "null factor");
    if (!(bound >= 0.0) || bound > 1.0) return fail(CULIPX_INVALID_ARG, "culipx_factor_set_pivot_fp64: bound not in [0, 1]");
    f->pivot_fp64 = bound;
    return CULIPX_OK;
}

CULIPX_API int culipx_prec_apply(culipx_factor f, int stage, const void* d_b, void* d_x)
{
    if (!f) return fail(CULIPX_INVALID_ARG, "null factor");
    GUARD_BEGIN
    CULIPX_TRY(use_device(f->pat->handle));
    return prec_apply(f, stage, d_b, d_x, f->pat->handle->stream);
    GUARD_END
}

CULIPX_API int culipx_csr_create(culipx_handle h, int m, int n, long long nnz, const int* d_rowptr,
                                 const int* d_colidx, const void* d_val, int precision, int explicit_transpose,
                                 culipx_csr* out)
{
    if (!h || !out || m < 0 || n < 0 || nnz < 0 || (nnz > 0 && (!d_colidx || !d_val)) || !d_rowptr)
        return fail(CULIPX_INVALID_ARG, "culipx_csr_create: bad arguments");
    if (h->device < 0) return fail(CULIPX_INVALID_ARG, "culipx_csr_create: host-only handle");
    if (precision != CULIPX_F64 && precision != CULIPX_F32)
        return fail(CULIPX_INVALID_ARG, "culipx_csr_create: bad precision");
    GUARD_BEGIN
    CULIPX_TRY(use_device(h));
    auto* A = new culipx_csr_t();
    A->h = h;
    A->m = m;
    A->n = n;
    A->nnz = nnz;
    A->rowptr = d_rowptr;
    A->colidx = d_colidx;
    A->val = d_val;
    A->precision = precision;
    if (explicit_transpose) {
        const int st = csr_build_transpose(A);
        if (st) { delete A; return st; }
    }
    handle_retain(h);
    *out = A;
    return CULIPX_OK;
    GUARD_END
}

CULIPX_API int culipx_kkt_assembly_create(culipx_handle h, int m, int n, long long nnz_a, const int* d_rowptr,
                                          const int* d_colidx, culipx_kkt_assembly* out)
{
    if (!h || !out) return fail(CULIPX_INVALID_ARG, "culipx_kkt_assembly_create: null argument");
    GUARD_BEGIN
    CULIPX_TRY(use_device(h));
    KktAssembly* K = nullptr;
    CULIPX_TRY(kkt_assembly_create(h, m, n, nnz_a, d_rowptr, d_colidx, &K));
    handle_retain(h);
    *out = static_cast<culipx_kkt_assembly>(K);
    return CULIPX_OK;
    GUARD_END
}

CULIPX_API int culipx_kkt_assembly_destroy(culipx_kkt_assembly K)
{
    if (K) {
        culipx_handle_t* h = K->handle;
        set_device_of(h);
        delete static_cast<KktAssembly*>(K);
        handle_release(h);
    }
    return CULIPX_OK;
}

CULIPX_API int culipx_kkt_assembly_size(culipx_kkt_assembly K, int* N, long long* nnz_k)
{
    if (!K) return fail(CULIPX_INVALID_ARG, "null plan");
    if (N) *N = K->n + K->m;
    if (nnz_k) *nnz_k = K->nnz_k;
    return CULIPX_OK;
}

CULIPX_API int culipx_kkt_assembly_structure(culipx_kkt_assembly K, const int** d_rowptr, const int** d_colidx)
{
    if (!K) return fail(CULIPX_INVALID_ARG, "null plan");
    if (d_rowptr) *d_rowptr = K->rowptr.as<int>();
    if (d_colidx) *d_colidx = K->colidx.as<int>();
    return CULIPX_OK;
}

CULIPX_API int culipx_kkt_assembly_export(culipx_kkt_assembly K, int* h_rowptr, int* h_colidx)
{
    if (!K || !h_rowptr || !h_colidx) return fail(CULIPX_INVALID_ARG, "culipx_kkt_assembly_export: null argument");
    GUARD_BEGIN
    CULIPX_TRY(use_device(K->handle));
    const size_t N = (size_t)K->n + K->m;
    CULIPX_CUDA(cudaMemcpy(h_rowptr, K->rowptr.get(), (N + 1) * sizeof(int), cudaMemcpyDeviceToHost));
    if (K->nnz_k > 0)
        CULIPX_CUDA(cudaMemcpy(h_colidx, K->colidx.get(), K->nnz_k * sizeof(int), cudaMemcpyDeviceToHost));
    return CULIPX_OK;
    GUARD_END
}

CULIPX_API int culipx_kkt_assemble(culipx_kkt_assembly K, const double* d_aval, const double* d_x, const double* d_s,
                                   const double* d_d, double delta, double gamma, int precision, void* d_kval)
{
    if (!K) return fail(CULIPX_INVALID_ARG, "culipx_kkt_assemble: null plan");
    GUARD_BEGIN
    CULIPX_TRY(use_device(K->handle));
    return kkt_assembly_values(K, d_aval, d_x, d_s, d_d, delta, gamma, precision, d_kval);
    GUARD_END
}

CULIPX_API int culipx_permute_create(culipx_handle h, int n, long long nnz, const int* d_rowptr,
                                     const int* d_colidx, const int* h_row_perm, const int* h_col_perm,
                                     int perm_is_old_to_new, culipx_permute* out)
{
    if (!h || !out) return fail(CULIPX_INVALID_ARG, "culipx_permute_create: null argument");
    GUARD_BEGIN
    CULIPX_TRY(use_device(h));
    PermutePlan* p = nullptr;
    CULIPX_TRY(permute_plan_create(h, n, nnz, d_rowptr, d_colidx, h_row_perm, h_col_perm, perm_is_old_to_new, &p));
    handle_retain(h);
    *out = static_cast<culipx_permute>(p);
    return CULIPX_OK;
    GUARD_END
}

CULIPX_API int culipx_permute_destroy(culipx_permute p)
{
    if (p) {
        culipx_handle_t* h = p->handle;
        set_device_of(h);
        delete p;
        handle_release(h);
    }
    return CULIPX_OK;
}

CULIPX_API int culipx_permute_structure(culipx_permute p, const int** d_rowptr, const int** d_colidx)
{
    if (!p) return fail(CULIPX_INVALID_ARG, "null plan");
    if (d_rowptr) *d_rowptr = p->rowptr.as<int>();
    if (d_colidx) *d_colidx = p->colidx.as<int>();
    return CULIPX_OK;
}

CULIPX_API int culipx_permute_export(culipx_permute p, int* h_rowptr, int* h_colidx)
{
    if (!p) return fail(CULIPX_INVALID_ARG, "null plan");
    GUARD_BEGIN
    CULIPX_TRY(use_device(p->handle));
    CULIPX_CUDA(cudaStreamSynchronize(p->handle->stream));
    if (h_rowptr)
        CULIPX_CUDA(cudaMemcpy(h_rowptr, p->rowptr.get(), (size_t)(p->n + 1) * sizeof(int), cudaMemcpyDeviceToHost));
    if (h_colidx && p->nnz)
        CULIPX_CUDA(cudaMemcpy(h_colidx, p->colidx.get(), (size_t)p->nnz * sizeof(int), cudaMemcpyDeviceToHost));
    return CULIPX_OK;
    GUARD_END
}

CULIPX_API int culipx_permute_apply(culipx_permute p, int precision, const void* d_val, const void* d_row_scale,
                                    const void* d_col_scale, int scale_before_match, void* d_out)
{
    if (!p) return fail(CULIPX_INVALID_ARG, "null plan");
    GUARD_BEGIN
    CULIPX_TRY(use_device(p->handle));
    return permute_plan_apply(p, precision, d_val, d_row_scale, d_col_scale, scale_before_match, d_out);
    GUARD_END
}

CULIPX_API int culipx_csr_destroy(culipx_csr A)
{
    if (A) {
        culipx_handle_t* h = A->h;
        set_device_of(h);
        delete A;
        handle_release(h);
    }
    return CULIPX_OK;
}

CULIPX_API int culipx_csr_set_format(culipx_csr A, int format)
{
    if (!A) return fail(CULIPX_INVALID_ARG, "null operator");
    if (format != CULIPX_FMT_CSR && format != CULIPX_FMT_SELL)
        return fail(CULIPX_INVALID_ARG, "culipx_csr_set_format: bad format %d", format);
    GUARD_BEGIN
    CULIPX_TRY(use_device(A->h));
    if (format == CULIPX_FMT_CSR) {
        A->sell = Sell();
        return CULIPX_OK;
    }
    return csr_build_sell(A);
    GUARD_END
}

CULIPX_API int culipx_csr_refresh(culipx_csr A)
{
    if (!A) return fail(CULIPX_INVALID_ARG, "null operator");
    GUARD_BEGIN
    CULIPX_TRY(use_device(A->h));
    return csr_refresh_sell(A, A->h->stream);
    GUARD_END
}

CULIPX_API int culipx_spmv(culipx_csr A, const void* d_x, void* d_y, double alpha, double beta, int transpose)
{
    if (!A) return fail(CULIPX_INVALID_ARG, "null operator");
    GUARD_BEGIN
    CULIPX_TRY(use_device(A->h));
    return csr_spmv(A, d_x, d_y, alpha, beta, transpose, A->h->stream);
    GUARD_END
}

CULIPX_API int culipx_sqmr_solve(culipx_handle h, culipx_csr A, culipx_factor M, const double* d_b, double* d_x,
                                 double tol, int max_it, double* residual, int* iterations)
{
    if (!h) return fail(CULIPX_INVALID_ARG, "null handle");
    if (h->device < 0) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve: host-only handle");
    GUARD_BEGIN
    CULIPX_TRY(use_device(h));
    return sqmr_solve(h, A, M, d_b, d_x, tol, max_it, residual, iterations, h->sqmr);
    GUARD_END
}

CULIPX_API int culipx_sqmr_profile(culipx_handle h, int enable)
{
    if (!h) return fail(CULIPX_INVALID_ARG, "null handle");
    h->sqmr->profile = enable != 0;
    return CULIPX_OK;
}

CULIPX_API int culipx_sqmr_set_wait_skew(culipx_handle h, unsigned long long skew)
{
    if (!h || !h->sqmr) return fail(CULIPX_INVALID_ARG, "null handle");
    h->sqmr->wait_skew = skew;
    return CULIPX_OK;
}

CULIPX_API int culipx_sqmr_phase_times(culipx_handle h, double* out_us, int iterations)
{
    if (!h || !out_us || iterations < 0) return fail(CULIPX_INVALID_ARG, "bad argument");
    if (!h->sqmr->profile || !h->sqmr->ts.get())
        return fail(CULIPX_INVALID_ARG, "culipx_sqmr_phase_times: profiling was not enabled for the last solve");
    CULIPX_TRY(use_device(h));
    const int its = iterations < 64 ? iterations : 64;
    unsigned long long ts[64 * 8];
    CULIPX_CUDA(cudaStreamSynchronize(h->stream));
    CULIPX_CUDA(cudaMemcpy(ts, h->sqmr->ts.get(), sizeof(ts), cudaMemcpyDeviceToHost));
    // per iteration: P1 (v+, ||v+||, first U level), the other U levels, the
    // first U' level (with the p / x update), the other U' levels with the
    // final reduction, 0, total; stamps: 0 start, 1 after P1, 2 after P2,
    // 4 after the first U' level (if there are two or more), 3 end
    for (int i = 0; i < its; ++i) {
        const unsigned long long* t = ts + i * 8;
        const unsigned long long next = (i + 1 < 64 && ts[(i + 1) * 8]) ? ts[(i + 1) * 8] : t[3];
        const unsigned long long mid = t[4] ? t[4] : t[3];
        const double d[6] = {(t[1] - t[0]) * 1e-3, (t[2] - t[1]) * 1e-3, (mid - t[2]) * 1e-3,
                             (t[3] - mid) * 1e-3, 0.0, (next - t[0]) * 1e-3};
        for (int k = 0; k < 6; ++k) out_us[i * 6 + k] = t[3] ? d[k] : 0.0;
    }
    return CULIPX_OK;
}

CULIPX_API int culipx_batch_create(culipx_pattern p, int num_systems, const int* h_row_offsets,
                                   culipx_batch* out)
{
    if (!p || !out) return fail(CULIPX_INVALID_ARG, "culipx_batch_create: null argument");
    if (p->handle->device < 0) return fail(CULIPX_INVALID_ARG, "culipx_batch_create: host-only handle");
    GUARD_BEGIN
    CULIPX_TRY(use_device(p->handle));
    Batch* b = nullptr;
    CULIPX_TRY(batch_create(p->handle, p, num_systems, h_row_offsets, &b));
    pattern_retain(p);
    b->pat_ref = p;
    *out = static_cast<culipx_batch>(b);
    return CULIPX_OK;
    GUARD_END
}

CULIPX_API int culipx_batch_destroy(culipx_batch b)
{
    if (b) {
        Pattern* p = b->pat_ref;
        set_device_of(b->h);
        delete b;
        pattern_release(p);
    }
    return CULIPX_OK;
}

CULIPX_API int culipx_batch_sqmr_solve(culipx_batch b, culipx_csr A, culipx_factor M, const double* d_b, double* d_x,
                                       double tol, int max_it, double* h_residual, int* h_iterations, int* h_status)
{
    if (!b) return fail(CULIPX_INVALID_ARG, "null batch");
    GUARD_BEGIN
    CULIPX_TRY(use_device(b->h));
    return batch_sqmr_solve(b, A, M, d_b, d_x, tol, max_it, h_residual, h_iterations, h_status, b->h->sqmr);
    GUARD_END
}

CULIPX_API int culipx_batch_factor_solve_graph(culipx_batch b, culipx_csr A, culipx_factor M, const void* d_vals,
                                               int pivot, double threshold, const double* d_b, double* d_x, double tol,
                                               int max_it, double* h_residual, int* h_iterations, int* h_status)
{
    if (!b) return fail(CULIPX_INVALID_ARG, "null batch");
    GUARD_BEGIN
    CULIPX_TRY(use_device(b->h));
    return batch_factor_solve_graph(b, A, M, d_vals, pivot, threshold, d_b, d_x, tol, max_it, h_residual,
                                    h_iterations, h_status);
    GUARD_END
}

CULIPX_API int culipx_sqmr_solve_multi(culipx_handle h, culipx_csr A, culipx_factor M, int nrhs, const double* d_B,
                                       double* d_X, double tol, int max_it, double* h_residual, int* h_iterations,
                                       int* h_status)
{
    if (!h) return fail(CULIPX_INVALID_ARG, "null handle");
    GUARD_BEGIN
    CULIPX_TRY(use_device(h));
    return sqmr_solve_multi(h, A, M, nrhs, d_B, d_X, tol, max_it, h_residual, h_iterations, h_status, h->sqmr);
    GUARD_END
}

CULIPX_API int culipx_sqmr_refine_multi(culipx_handle h, culipx_csr A, culipx_factor M, int nrhs, const double* d_B,
                                        double* d_X, double tol, double inner_tol, int inner_max_it, int max_refine,
                                        double* h_relres, int* h_iterations, int* h_steps, int* h_status)
{
    if (!h) return fail(CULIPX_INVALID_ARG, "null handle");
    GUARD_BEGIN
    CULIPX_TRY(use_device(h));
    return sqmr_refine_multi(h, A, M, nrhs, d_B, d_X, tol, inner_tol, inner_max_it, max_refine, h_relres,
                             h_iterations, h_steps, h_status, h->sqmr);
    GUARD_END
}

CULIPX_API int culipx_sqmr_solve_many(culipx_handle h, int num, const culipx_csr* A, const culipx_factor* M,
                                      const double* const* d_b, double* const* d_x, double tol, int max_it,
                                      double* h_residual, int* h_iterations, int* h_status)
{
    if (!h) return fail(CULIPX_INVALID_ARG, "null handle");
    GUARD_BEGIN
    CULIPX_TRY(use_device(h));
    std::vector<Csr*> a(num > 0 ? num : 0);
    std::vector<Factor*> m(num > 0 ? num : 0);
    for (int k = 0; k < num; ++k) {
        a[k] = A ? A[k] : nullptr;
        m[k] = M ? M[k] : nullptr;
    }
    return sqmr_solve_many(h, num, a.data(), m.data(), d_b, d_x, tol, max_it, h_residual, h_iterations, h_status,
                           h->sqmr);
    GUARD_END
}

CULIPX_API int culipx_server_create(int device, long long memory_budget, int slots, int max_batch, double tol,
                                    int max_it, culipx_server* out)
{
    GUARD_BEGIN
    Server* s = nullptr;
    CULIPX_TRY(server_create(device, memory_budget, slots, max_batch, tol, max_it, &s));
    *out = static_cast<culipx_server>(s);
    return CULIPX_OK;
    GUARD_END
}

CULIPX_API int culipx_server_destroy(culipx_server s)
{
    delete s;
    return CULIPX_OK;
}

CULIPX_API int culipx_server_add_pattern(culipx_server s, int n, const int* h_rowptr, const int* h_colidx,
                                         int num_blocks, const int* h_block_starts, int precision, int* pattern_id)
{
    GUARD_BEGIN
    return server_add_pattern(s, n, h_rowptr, h_colidx, num_blocks, h_block_starts, precision, pattern_id);
    GUARD_END
}

CULIPX_API int culipx_server_submit(culipx_server s, int pattern_id, const double* h_vals, int nrhs,
                                    const double* h_b, int* request_id)
{
    GUARD_BEGIN
    return server_submit(s, pattern_id, h_vals, nrhs, h_b, request_id);
    GUARD_END
}

CULIPX_API int culipx_server_progress(culipx_server s, int wait, int* completed)
{
    GUARD_BEGIN
    return server_progress(s, wait, completed);
    GUARD_END
}

CULIPX_API int culipx_server_result(culipx_server s, int request_id, double* h_x, int* h_iterations, int* h_status,
                                    double* latency_ms)
{
    GUARD_BEGIN
    return server_result(s, request_id, h_x, h_iterations, h_status, latency_ms);
    GUARD_END
}

CULIPX_API int culipx_server_release(culipx_server s, int request_id)
{
    GUARD_BEGIN
    return server_release(s, request_id);
    GUARD_END
}

CULIPX_API int culipx_server_stats(culipx_server s, long long* stats8)
{
    return server_stats(s, stats8);
}

CULIPX_API int culipx_server_set_large_rows(culipx_server s, int rows)
{
    return server_set_large_rows(s, rows);
}

CULIPX_API int culipx_ldu_create(culipx_handle h, int n, const int* d_rowptr, const int* d_colidx, const double* d_val,
                                 const double* d_tri, const int* d_is_piv, const int* d_perm, const double* d_scale,
                                 culipx_ldu* out)
{
    if (!h || !out) return fail(CULIPX_INVALID_ARG, "culipx_ldu_create: null argument");
    if (h->device < 0) return fail(CULIPX_INVALID_ARG, "culipx_ldu_create: host-only handle");
    GUARD_BEGIN
    CULIPX_TRY(use_device(h));
    Ldu* P = nullptr;
    CULIPX_TRY(ldu_create(h, n, d_rowptr, d_colidx, d_val, d_tri, d_is_piv, d_perm, d_scale, &P));
    handle_retain(h);
    *out = static_cast<culipx_ldu>(P);
    return CULIPX_OK;
    GUARD_END
}

CULIPX_API int culipx_ldu_apply(culipx_ldu P, int stage, const double* d_b, double* d_x)
{
    if (!P) return fail(CULIPX_INVALID_ARG, "null preconditioner");
    GUARD_BEGIN
    CULIPX_TRY(use_device(P->h));
    return ldu_apply(P, stage, d_b, d_x, P->h->stream);
    GUARD_END
}

CULIPX_API int culipx_sqmr_solve_ldu(culipx_handle h, culipx_csr A, culipx_ldu P, const double* d_b, double* d_x,
                                     double tol, int max_it, double* residual, int* iterations)
{
    if (!h) return fail(CULIPX_INVALID_ARG, "null handle");
    GUARD_BEGIN
    CULIPX_TRY(use_device(h));
    return sqmr_solve_ldu(h, A, P, d_b, d_x, tol, max_it, residual, iterations, h->sqmr);
    GUARD_END
}

CULIPX_API int culipx_ldu_destroy(culipx_ldu P)
{
    if (P) {
        culipx_handle_t* h = P->h;
        set_device_of(h);
        delete P;
        handle_release(h);
    }
    return CULIPX_OK;
}

CULIPX_API int culipx_kkt_operator_create(culipx_handle h, int kind, int m, int n, long long nnz, const int* d_rowptr,
                                         const int* d_colidx, const double* d_val, const double* d_d, double delta,
                                         int num_ix, const int* d_ix, culipx_kkt_operator* out)
{
    if (!h || !out) return fail(CULIPX_INVALID_ARG, "culipx_kkt_operator_create: null argument");
    if (h->device < 0) return fail(CULIPX_INVALID_ARG, "culipx_kkt_operator_create: host-only handle");
    GUARD_BEGIN
    CULIPX_TRY(use_device(h));
    KktOperator* op = nullptr;
    CULIPX_TRY(kkt_operator_create(h, kind, m, n, nnz, d_rowptr, d_colidx, d_val, d_d, delta, num_ix, d_ix, &op));
    handle_retain(h);
    *out = static_cast<culipx_kkt_operator>(op);
    return CULIPX_OK;
    GUARD_END
}

CULIPX_API int culipx_kkt_operator_multiply(culipx_kkt_operator op, const double* d_x, double* d_y, double alpha,
                                           double beta)
{
    if (!op) return fail(CULIPX_INVALID_ARG, "null operator");
    GUARD_BEGIN
    CULIPX_TRY(use_device(op->h));
    return kkt_operator_multiply(op, d_x, d_y, alpha, beta);
    GUARD_END
}

CULIPX_API int culipx_kkt_operator_destroy(culipx_kkt_operator op)
{
    if (op) {
        culipx_handle_t* h = op->h;
        set_device_of(h);
        delete op;
        handle_release(h);
    }
    return CULIPX_OK;
}

CULIPX_API int culipx_tune_kkt_block(culipx_handle h, int n, int m, const int* h_rowptr, const int* h_colidx,
                                     const double* d_vals, const double* d_b, int precision, const int* candidates,
                                     int num_candidates, double tol, int max_it, int* best_block, double* h_ms,
                                     int* h_iterations, int* h_status, double* h_residual)
{
    if (!h) return fail(CULIPX_INVALID_ARG, "null handle");
    GUARD_BEGIN
    CULIPX_TRY(use_device(h));
    return tune_kkt_block(h, n, m, h_rowptr, h_colidx, d_vals, d_b, precision, candidates, num_candidates, tol,
                          max_it, best_block, h_ms, h_iterations, h_status, h_residual);
    GUARD_END
}

CULIPX_API int culipx_server_set_refine(culipx_server s, int max_refine, double inner_tol)
{
    return server_set_refine(s, max_refine, inner_tol);
}

CULIPX_API int culipx_server_launch_count(culipx_server s, long long* count)
{
    return server_launch_count(s, count);
}

CULIPX_API int culipx_batch_sqmr_refine(culipx_batch b, culipx_csr A, culipx_factor M, const double* d_b,
                                        double* d_x, double tol, double inner_tol, int inner_max_it, int max_refine,
                                        double* h_relres, int* h_iterations, int* h_steps, int* h_status)
{
    if (!b) return fail(CULIPX_INVALID_ARG, "null batch");
    GUARD_BEGIN
    CULIPX_TRY(use_device(b->h));
    return batch_sqmr_refine(b, A, M, d_b, d_x, tol, inner_tol, inner_max_it, max_refine, h_relres, h_iterations,
                             h_steps, h_status, b->h->sqmr);
    GUARD_END
}

CULIPX_API int culipx_sqmr_refine(culipx_handle h, culipx_csr A, culipx_factor M, const double* d_b, double* d_x,
                                  double tol, double inner_tol, int inner_max_it, int max_refine, double* relres,
                                  int* iterations, int* steps)
{
    if (!h) return fail(CULIPX_INVALID_ARG, "null handle");
    GUARD_BEGIN
    CULIPX_TRY(use_device(h));
    return sqmr_refine(h, A, M, d_b, d_x, tol, inner_tol, inner_max_it, max_refine, relres, iterations, steps,
                       h->sqmr);
    GUARD_END
}

CULIPX_API int culipx_sqmr_solve_noalloc(culipx_handle h, culipx_csr A, culipx_factor M, const double* d_b,
                                         double* d_x, double tol, int max_it, double* residual, int* iterations)
{
    if (!h) return fail(CULIPX_INVALID_ARG, "null handle");
    if (h->device < 0) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_noalloc: host-only handle");
    GUARD_BEGIN
    CULIPX_TRY(use_device(h));
    return sqmr_solve_noalloc(h, A, M, d_b, d_x, tol, max_it, residual, iterations);
    GUARD_END
}

}  // extern "C"
