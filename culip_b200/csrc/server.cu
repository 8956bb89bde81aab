// Request server for streams of KKT solves (no counterpart in the reference,
// whose driver solves one system per process run, apps/block_ildlt).
//
// A request is one IPM iteration on a registered sparsity pattern: new
// values of K and 1..k right-hand sides.  The server
//   * analyses each pattern once (symbolic phase, device mirror, K's
//     structure on the device) and keeps a pool of factor objects per
//     pattern, reused across requests;
//   * admits queued requests in arrival order while the device-memory budget
//     allows (request buffers come from the stream-ordered allocator, so
//     admission and release never synchronize the device);
//   * runs admitted requests as a batch on one of several slots, each with
//     its own stream and workspace: per request the values' upload and the
//     numeric factor, then the solves; results come back through pinned
//     buffers.  A batch holds requests of one class, the class of the
//     oldest queued request, in arrival order (requests of the other class
//     keep their places in the queue):
//       - small patterns (n < large_rows): one CTA per request and group
//         of up to 4 of its right-hand sides (k_sqmr_many, one launch per
//         factor precision and group size);
//       - large patterns: per request the whole-GPU cooperative solver,
//         its right-hand sides in groups of up to 4 per launch (one CTA per
//         system would leave a large system to a single SM for its whole
//         solve).  A large batch runs alone on the device: it starts when no
//         other batch runs, and none starts beside it;
//   * keeps up to `slots` small batches in flight, so requests that arrive
//     while others run are admitted into the next slot and overlap on the
//     device.
// Latency is measured from submit to the progress() call that sees the
// batch's completion event.
#include "server.h"
#include "factor.h"
#include "pattern.h"
#include "kernels_common.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

namespace culipx {

namespace {

__global__ void k_to_f32(const double* __restrict__ in, float* __restrict__ out, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) out[i] = (float)in[i];
}

// one right-hand side of a refinement round: v += a (if a), r = b - K v, ||r||^2
struct ResJob {
    const int* rowptr;
    const int* colidx;
    const double* val;
    const double* b;
    const double* a;
    double* v;
    double* r;
    long long n;
};

constexpr int kResT = 256;
constexpr int kRefinePatience = 2;  // corrections in a row without a smaller residual that stop a right-hand side

__global__ void k_add_corrections(const ResJob* __restrict__ jobs, int num)
{
    for (int j = blockIdx.x; j < num; j += gridDim.x) {
        const ResJob J = jobs[j];
        if (J.a)
            for (long long i = threadIdx.x; i < J.n; i += kResT) J.v[i] += J.a[i];
    }
}

// one CTA per right-hand side; the sum of squares in a fixed order
__global__ void k_residuals(const ResJob* __restrict__ jobs, int num, double* __restrict__ sumsq)
{
    __shared__ double sh[kResT / 32];
    for (int j = blockIdx.x; j < num; j += gridDim.x) {
        const ResJob J = jobs[j];
        double t = 0.0;
        for (long long i = threadIdx.x; i < J.n; i += kResT) {
            double acc = 0.0;
            for (int k = __ldg(J.rowptr + i); k < __ldg(J.rowptr + i + 1); ++k)
                acc = fma_rn(__ldg(J.val + k), J.v[__ldg(J.colidx + k)], acc);
            const double ri = J.b[i] - acc;
            J.r[i] = ri;
            t = fma_rn(ri, ri, t);
        }
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = t;
        __syncthreads();
        if (threadIdx.x == 0) {
            double u = 0.0;
            for (int w = 0; w < kResT / 32; ++w) u += sh[w];
            sumsq[j] = u;
        }
        __syncthreads();
    }
}

double now_ms()
{
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

long long request_bytes(const ServerPattern& sp, int nrhs, bool refine)
{
    const long long n = sp.n;
    long long b = sp.nnz * 8 + 2 * n * nrhs * 8 + (long long)(7 * n + 8) * nrhs * 8 + 4096;
    if (refine) b += 3 * n * nrhs * 8;
    if (sp.precision == CULIPX_F32) b += sp.nnz * 4;
    return b;
}

}  // namespace

int server_create(int device, long long budget, int slots, int max_batch, double tol, int max_it, Server** out)
{
    if (!out || slots < 1 || slots > 8 || max_batch < 1 || !(tol >= 0.0) || max_it < 0)
        return fail(CULIPX_INVALID_ARG, "culipx_server_create: bad argument");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return fail(CULIPX_INVALID_ARG, "culipx_server_create: bad device %d", device);
    }
    CULIPX_CUDA(cudaSetDevice(device));
    {
        // keep freed request buffers in the process's pool (no OS round trips)
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            unsigned long long keep = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
    }
    auto* s = new culipx_server_t();
    s->device = device;
    s->budget = budget;
    s->max_batch = max_batch;
    s->tol = tol;
    s->max_it = max_it;
    s->base = new culipx_handle_t();
    s->base->device = device;
    s->base->sqmr = new Sqmr();
    if (cudaEventCreate(&s->base->ev_start) != cudaSuccess || cudaEventCreate(&s->base->ev_stop) != cudaSuccess) {
        delete s;
        return fail(CULIPX_CUDA_ERROR, "culipx_server_create: event creation failed");
    }
    s->slots.resize(slots);
    for (auto& sl : s->slots) {
        sl.h = new culipx_handle_t();
        sl.h->device = device;
        sl.h->sqmr = new Sqmr();
        if (cudaStreamCreateWithFlags(&sl.h->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreate(&sl.h->ev_start) != cudaSuccess || cudaEventCreate(&sl.h->ev_stop) != cudaSuccess) {
            delete s;
            return fail(CULIPX_CUDA_ERROR, "culipx_server_create: stream / event creation failed");
        }
    }
    *out = s;
    return CULIPX_OK;
}

Server::~Server()
{
    cudaSetDevice(device);
    for (auto& sl : slots) {
        if (sl.h && sl.h->stream) cudaStreamSynchronize(sl.h->stream);
    }
    for (auto& r : requests)
        for (void* p : {r.second.d_vals, r.second.d_vals32, r.second.d_b, r.second.d_x, r.second.d_r, r.second.d_d,
                        r.second.d_best})
            if (p) cudaFree(p);
    for (auto& sp : patterns) {
        for (Factor* f : sp.free_factors) delete static_cast<culipx_factor_t*>(f);
        delete static_cast<culipx_pattern_t*>(sp.pat);
    }
    for (auto& sl : slots) {
        if (sl.out_host) cudaFreeHost(sl.out_host);
        if (sl.x_host) cudaFreeHost(sl.x_host);
        if (sl.res_host) cudaFreeHost(sl.res_host);
        if (sl.done) cudaEventDestroy(sl.done);
        sl.jobs.release();  // charged to sl.h, released before it
        if (sl.h) {
            delete sl.h->sqmr;
            if (sl.h->stream) cudaStreamDestroy(sl.h->stream);
            if (sl.h->ev_start) cudaEventDestroy(sl.h->ev_start);
            if (sl.h->ev_stop) cudaEventDestroy(sl.h->ev_stop);
            delete sl.h;
        }
    }
    if (base) {
        delete base->sqmr;
        if (base->ev_start) cudaEventDestroy(base->ev_start);
        if (base->ev_stop) cudaEventDestroy(base->ev_stop);
        delete base;
    }
}

int server_add_pattern(Server* s, int n, const int* rowptr, const int* colidx, int num_blocks, const int* block_starts,
                       int precision, int* pattern_id)
{
    if (!s || !pattern_id) return fail(CULIPX_INVALID_ARG, "culipx_server_add_pattern: null argument");
    CULIPX_CUDA(cudaSetDevice(s->device));
    Pattern* p = nullptr;
    CULIPX_TRY(analyze_pattern(s->base, n, rowptr, colidx, num_blocks, block_starts, 0, 1.0, precision, &p));
    ServerPattern sp;
    sp.pat = p;
    sp.n = n;
    sp.nnz = p->nnz;
    sp.precision = precision;
    int st = sp.d_rowptr.upload(s->base, rowptr, (size_t)(n + 1) * sizeof(int));
    if (st == CULIPX_OK) st = sp.d_colidx.upload(s->base, colidx, (size_t)std::max<long long>(sp.nnz, 1) * sizeof(int));
    if (st != CULIPX_OK) {
        delete static_cast<culipx_pattern_t*>(p);
        return st;
    }
    s->patterns.push_back(std::move(sp));
    *pattern_id = (int)s->patterns.size() - 1;
    return CULIPX_OK;
}

int server_submit(Server* s, int pid, const double* vals, int nrhs, const double* b, int* request_id)
{
    if (!s || !vals || !b || !request_id || nrhs < 1) return fail(CULIPX_INVALID_ARG, "culipx_server_submit: bad argument");
    if (pid < 0 || pid >= (int)s->patterns.size()) return fail(CULIPX_INVALID_ARG, "culipx_server_submit: unknown pattern %d", pid);
    const ServerPattern& sp = s->patterns[pid];
    if (s->budget > 0 && request_bytes(sp, nrhs, s->max_refine > 0) > s->budget)
        return fail(CULIPX_OOM, "culipx_server_submit: the request alone exceeds the memory budget");
    ServerRequest r;
    r.id = s->next_id++;
    r.pid = pid;
    r.nrhs = nrhs;
    r.vals.assign(vals, vals + sp.nnz);
    r.b.assign(b, b + (size_t)sp.n * nrhs);
    r.t_submit = now_ms();
    const int id = r.id;
    s->queue.push_back(id);
    s->requests.emplace(id, std::move(r));
    *request_id = id;
    return CULIPX_OK;
}

long long Server::fixed_bytes() const
{
    long long t = 0;
    for (const auto& sp : patterns) t += sp.pat->device_bytes + sp.d_rowptr.bytes() + sp.d_colidx.bytes() + sp.pool_bytes;
    return t;
}

int server_launch_count(Server* s, long long* out)
{
    if (!s || !out) return fail(CULIPX_INVALID_ARG, "null argument");
    long long t = s->base->launches;
    for (const auto& sl : s->slots) t += sl.h->launches;
    *out = t;
    return CULIPX_OK;
}

int server_set_refine(Server* s, int max_refine, double inner_tol)
{
    if (!s || max_refine < 0 || !(inner_tol >= 0.0))
        return fail(CULIPX_INVALID_ARG, "culipx_server_set_refine: bad argument");
    s->max_refine = max_refine;
    s->inner_tol = inner_tol;
    return CULIPX_OK;
}

int server_set_large_rows(Server* s, int rows)
{
    if (!s || rows < 1) return fail(CULIPX_INVALID_ARG, "culipx_server_set_large_rows: bad argument");
    s->large_rows = rows;
    return CULIPX_OK;
}

namespace {

// requests per large batch: large batches are exclusive, so small requests
// queued behind them get the device back after a few
constexpr int kLargeBatch = 4;

// work units that keep every CTA of a batched launch busy (2 per SM)
constexpr int kManyUnits = 296;

int finish_slot(Server* s, ServerSlot& sl)
{
    const double t = now_ms();
    int k = 0;
    size_t xo = 0;
    for (int id : sl.reqs) {
        ServerRequest& r = s->requests.at(id);
        const ServerPattern& sp = s->patterns[r.pid];
        r.its.resize(r.nrhs);
        r.status.resize(r.nrhs);
        if (s->max_refine > 0 && (int)r.its_acc.size() == r.nrhs) {
            for (int c = 0; c < r.nrhs; ++c) {
                r.its[c] = r.its_acc[c];
                r.status[c] = r.broke[c]           ? CULIPX_BREAKDOWN
                              : r.rel[c] <= s->tol ? CULIPX_OK
                              : r.stalled[c]       ? CULIPX_STALLED
                                                   : CULIPX_MAXIT;
            }
        } else {
            many_results(r.nrhs, s->max_it, sl.out_host + (size_t)k * 8, nullptr, r.its.data(), r.status.data());
        }
        k += r.nrhs;
        r.x.assign(sl.x_host + xo, sl.x_host + xo + (size_t)sp.n * r.nrhs);
        xo += (size_t)sp.n * r.nrhs;
        r.t_done = t;
        r.state = 2;
        s->patterns[r.pid].free_factors.push_back(r.F);
        r.F = nullptr;
        s->in_use -= r.bytes;
        r.vals.clear();
        r.vals.shrink_to_fit();
        r.b.clear();
        r.b.shrink_to_fit();
        ++s->done;
    }
    sl.reqs.clear();
    sl.busy = false;
    sl.large = false;
    return CULIPX_OK;
}

// the batch's end on its stream: solutions to the pinned buffer, request
// buffers back to the pool, the completion event
int enqueue_end(Server* s, ServerSlot& sl)
{
    cudaStream_t st = sl.h->stream;
    size_t xo = 0;
    for (int id : sl.reqs) {
        ServerRequest& r = s->requests.at(id);
        const size_t nb = (size_t)s->patterns[r.pid].n * r.nrhs;
        // refined requests return their best iterates
        const void* src = r.d_best ? r.d_best : r.d_x;
        CULIPX_CUDA(cudaMemcpyAsync(sl.x_host + xo, src, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
        xo += nb;
        for (void** p : {&r.d_vals, &r.d_vals32, &r.d_b, &r.d_x, &r.d_r, &r.d_d, &r.d_best})
            if (*p) {
                CULIPX_CUDA(cudaFreeAsync(*p, st));
                *p = nullptr;
            }
    }
    CULIPX_CUDA(cudaEventRecord(sl.done, st));
    return CULIPX_OK;
}

// r = b - K x for the right-hand sides in sl.cols (after x += d when add),
// their sums of squares to the pinned buffer, then the completion event
int enqueue_residuals(Server* s, ServerSlot& sl, bool add)
{
    cudaStream_t st = sl.h->stream;
    const int num = (int)sl.cols.size();
    std::vector<ResJob> jobs(num);
    for (int i = 0; i < num; ++i) {
        ServerRequest& r = s->requests.at(sl.cols[i].first);
        const size_t c = sl.cols[i].second, n = s->patterns[r.pid].n;
        const Csr& A = sl.csrs[r.q];
        jobs[i] = ResJob{A.rowptr, A.colidx, static_cast<const double*>(A.val), static_cast<const double*>(r.d_b) + c * n,
                         add ? static_cast<const double*>(r.d_d) + c * n : nullptr, static_cast<double*>(r.d_x) + c * n,
                         static_cast<double*>(r.d_r) + c * n, (long long)n};
    }
    const size_t need = (size_t)num * (sizeof(ResJob) + sizeof(double)) + 64;
    if (sl.jobs.bytes() < need) CULIPX_TRY(sl.jobs.alloc(sl.h, 2 * need));
    ResJob* d_jobs = sl.jobs.as<ResJob>();
    double* d_sum = reinterpret_cast<double*>(d_jobs + num);
    CULIPX_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), (size_t)num * sizeof(ResJob), cudaMemcpyHostToDevice, st));
    if (add) {
        k_add_corrections<<<std::min(num, 148 * 8), kResT, 0, st>>>(d_jobs, num);
        sl.h->launches += 1;
        CULIPX_TRY(launch_check("k_add_corrections"));
    }
    k_residuals<<<std::min(num, 148 * 8), kResT, 0, st>>>(d_jobs, num, d_sum);
    sl.h->launches += 1;
    CULIPX_TRY(launch_check("k_residuals"));
    if (sl.res_cap < (size_t)num) {
        if (sl.res_host) cudaFreeHost(sl.res_host);
        sl.res_host = nullptr;
        CULIPX_CUDA(cudaMallocHost(&sl.res_host, (size_t)num * sizeof(double)));
        sl.res_cap = num;
    }
    CULIPX_CUDA(cudaMemcpyAsync(sl.res_host, d_sum, (size_t)num * sizeof(double), cudaMemcpyDeviceToHost, st));
    CULIPX_CUDA(cudaEventRecord(sl.done, st));
    return CULIPX_OK;
}

// A refinement round finished: take the last solves' iterations and the new
// residuals (the first round's is the plain solve's).  An iterate with the
// smallest residual so far is copied to best; kRefinePatience corrections in
// a row without a new smallest residual stop the right-hand side (stalled).
// Right-hand sides still above tol (and below max_refine corrections, not
// stalled, without breakdown) get a correction d = SQMR(K, M, r, inner_tol),
// x += d and a new residual; otherwise the batch ends, returning the best
// iterates.
int refine_step(Server* s, ServerSlot& sl)
{
    std::vector<std::pair<int, int>> next;
    for (size_t i = 0; i < sl.cols.size(); ++i) {
        ServerRequest& r = s->requests.at(sl.cols[i].first);
        const int c = sl.cols[i].second;
        const size_t n = s->patterns[r.pid].n;
        const double* o = sl.out_host + 8 * i;
        r.its_acc[c] += (int)o[1];
        if (o[2] != 0.0) r.broke[c] = 1;
        const double rel = r.bnorm[c] > 0.0 ? std::sqrt(sl.res_host[i]) / r.bnorm[c] : 0.0;
        if (!std::isfinite(rel)) r.broke[c] = 1;
        if (r.steps[c] == 0 || (!r.broke[c] && rel < r.rel[c])) {
            r.rel[c] = rel;
            r.fails[c] = 0;
            CULIPX_CUDA(cudaMemcpyAsync(static_cast<double*>(r.d_best) + c * n, static_cast<double*>(r.d_x) + c * n,
                                        n * sizeof(double), cudaMemcpyDeviceToDevice, sl.h->stream));
        } else if (!r.broke[c] && ++r.fails[c] >= kRefinePatience) {
            r.stalled[c] = 1;
        }
        if (!r.broke[c] && !r.stalled[c] && r.rel[c] > s->tol && r.steps[c] < s->max_refine)
            next.push_back(sl.cols[i]);
    }
    if (next.empty()) {
        sl.phase = 0;
        return enqueue_end(s, sl);
    }
    const int num = (int)next.size();
    std::vector<Csr*> As(num);
    std::vector<Factor*> Ms(num);
    std::vector<const double*> bs(num);
    std::vector<double*> xs(num);
    for (int i = 0; i < num; ++i) {
        ServerRequest& r = s->requests.at(next[i].first);
        const size_t c = next[i].second, n = s->patterns[r.pid].n;
        r.steps[c] += 1;
        As[i] = &sl.csrs[r.q];
        Ms[i] = r.F;
        bs[i] = static_cast<const double*>(r.d_r) + c * n;
        xs[i] = static_cast<double*>(r.d_d) + c * n;
    }
    if (sl.large) {
        for (int i = 0; i < num; ++i)
            CULIPX_TRY(sqmr_solve_multi_async(sl.h, As[i], Ms[i], 1, bs[i], xs[i], s->inner_tol, s->max_it, sl.h->sqmr,
                                              sl.out_host + (size_t)8 * i));
    } else {
        CULIPX_TRY(sqmr_solve_many_nr_async(sl.h, num, As.data(), Ms.data(), bs.data(), xs.data(), nullptr,
                                            s->inner_tol, s->max_it, sl.h->sqmr, sl.out_host));
    }
    sl.cols = next;
    return enqueue_residuals(s, sl, true);
}

int launch_slot(Server* s, ServerSlot& sl)
{
    cudaStream_t st = sl.h->stream;
    if (s->queue.empty()) return CULIPX_OK;
    for (const auto& o : s->slots)
        if (o.busy && o.large) return CULIPX_OK;  // a large batch has the device
    auto is_large = [&](int id) { return s->patterns[s->requests.at(id).pid].n >= s->large_rows; };
    const bool large = is_large(s->queue.front());
    if (large && s->running_slots() > 0) return CULIPX_OK;  // wait until the device is idle
    const int cap = large ? std::min(s->max_batch, kLargeBatch) : s->max_batch;
    // admit requests of the oldest request's class, in arrival order (those of
    // the other class keep their places), while the budget allows
    std::vector<int> admit;
    int systems = 0;
    std::deque<int> rest;
    while (!s->queue.empty()) {
        const int id = s->queue.front();
        s->queue.pop_front();
        if ((int)admit.size() >= cap || is_large(id) != large) {
            rest.push_back(id);
            continue;
        }
        ServerRequest& r = s->requests.at(id);
        const ServerPattern& sp = s->patterns[r.pid];
        const long long need = request_bytes(sp, r.nrhs, s->max_refine > 0);
        const long long fbytes = sp.free_factors.empty() ? sp.factor_bytes_estimate() : 0;
        const bool fits = s->budget <= 0 || s->fixed_bytes() + s->in_use + need + fbytes <= s->budget;
        // over the budget: wait for running batches to free memory (a request
        // that fits alone always runs once the device is idle)
        if (!fits && (!admit.empty() || s->running_slots() > 0)) {
            rest.push_back(id);
            while (!s->queue.empty()) {
                rest.push_back(s->queue.front());
                s->queue.pop_front();
            }
            break;
        }
        r.bytes = need;
        s->in_use += need;
        admit.push_back(r.id);
        systems += r.nrhs;
    }
    s->queue.swap(rest);
    if (admit.empty()) return CULIPX_OK;
    // pinned result buffers
    size_t xtot = 0;
    for (int id : admit) xtot += (size_t)s->patterns[s->requests.at(id).pid].n * s->requests.at(id).nrhs;
    if (sl.out_cap < systems) {
        if (sl.out_host) cudaFreeHost(sl.out_host);
        CULIPX_CUDA(cudaMallocHost(&sl.out_host, (size_t)systems * 8 * sizeof(double)));
        sl.out_cap = systems;
    }
    if (sl.x_cap < xtot) {
        if (sl.x_host) cudaFreeHost(sl.x_host);
        CULIPX_CUDA(cudaMallocHost(&sl.x_host, std::max<size_t>(xtot, 1) * sizeof(double)));
        sl.x_cap = xtot;
    }
    std::vector<Csr*> As;
    std::vector<Factor*> Ms;
    std::vector<const double*> bs;
    std::vector<double*> xs;
    sl.csrs.clear();
    sl.csrs.reserve(admit.size());
    for (int id : admit) {
        ServerRequest& r = s->requests.at(id);
        ServerPattern& sp = s->patterns[r.pid];
        if (sp.free_factors.empty()) {
            Factor* f = nullptr;
            CULIPX_TRY(factor_create(sp.pat, &f));
            sp.pool_bytes += sp.factor_bytes_estimate();
            r.F = f;
        } else {
            r.F = sp.free_factors.back();
            sp.free_factors.pop_back();
        }
        const size_t nv = (size_t)sp.nnz, nb = (size_t)sp.n * r.nrhs;
        CULIPX_CUDA(cudaMallocAsync(&r.d_vals, std::max<size_t>(nv, 1) * sizeof(double), st));
        CULIPX_CUDA(cudaMallocAsync(&r.d_b, nb * sizeof(double), st));
        CULIPX_CUDA(cudaMallocAsync(&r.d_x, nb * sizeof(double), st));
        if (s->max_refine > 0) {
            CULIPX_CUDA(cudaMallocAsync(&r.d_r, nb * sizeof(double), st));
            CULIPX_CUDA(cudaMallocAsync(&r.d_d, nb * sizeof(double), st));
            CULIPX_CUDA(cudaMallocAsync(&r.d_best, nb * sizeof(double), st));
            r.bnorm.assign(r.nrhs, 0.0);
            for (int c = 0; c < r.nrhs; ++c) {
                double t = 0.0;
                for (size_t i = 0; i < (size_t)sp.n; ++i) t += r.b[c * (size_t)sp.n + i] * r.b[c * (size_t)sp.n + i];
                r.bnorm[c] = std::sqrt(t);
            }
            r.rel.assign(r.nrhs, 1.0);
            r.steps.assign(r.nrhs, 0);
            r.its_acc.assign(r.nrhs, 0);
            r.broke.assign(r.nrhs, 0);
            r.stalled.assign(r.nrhs, 0);
            r.fails.assign(r.nrhs, 0);
        }
        r.q = (int)(sl.csrs.size());
        CULIPX_CUDA(cudaMemcpyAsync(r.d_vals, r.vals.data(), nv * sizeof(double), cudaMemcpyHostToDevice, st));
        CULIPX_CUDA(cudaMemcpyAsync(r.d_b, r.b.data(), nb * sizeof(double), cudaMemcpyHostToDevice, st));
        const void* fv = r.d_vals;
        if (sp.precision == CULIPX_F32) {
            CULIPX_CUDA(cudaMallocAsync(&r.d_vals32, std::max<size_t>(nv, 1) * sizeof(float), st));
            k_to_f32<<<148 * 4, 256, 0, st>>>(static_cast<const double*>(r.d_vals), static_cast<float*>(r.d_vals32),
                                              (long long)nv);
            fv = r.d_vals32;
        }
        // the factor runs on this slot's stream
        cudaStream_t keep = sp.pat->handle->stream;
        sp.pat->handle->stream = st;
        const int fs = factor_compute(r.F, fv, nullptr, CULIPX_PIV_BK, 0.0);
        sp.pat->handle->stream = keep;
        CULIPX_TRY(fs);
        sl.csrs.emplace_back();
        Csr& A = sl.csrs.back();
        A.h = sl.h;
        A.m = A.n = sp.n;
        A.nnz = sp.nnz;
        A.rowptr = sp.d_rowptr.as<int>();
        A.colidx = sp.d_colidx.as<int>();
        A.val = r.d_vals;
        A.precision = CULIPX_F64;
        r.state = 1;
    }
    if (large) {
        // whole-GPU solves, request after request on this stream; results in
        // request order
        int k = 0;
        for (size_t q = 0; q < admit.size(); ++q) {
            ServerRequest& r = s->requests.at(admit[q]);
            CULIPX_TRY(sqmr_solve_multi_async(sl.h, &sl.csrs[q], r.F, r.nrhs, static_cast<const double*>(r.d_b),
                                              static_cast<double*>(r.d_x), s->tol, s->max_it, sl.h->sqmr,
                                              sl.out_host + (size_t)k * 8));
            k += r.nrhs;
        }
        ++s->large_batches;
    }
    if (!large) {
        // one CTA per (request, group of 4 / 2 / 1 right-hand sides): the
        // group's right-hand sides share every factor and K load; results
        // land in request order
        std::vector<int> nrs;
        // group right-hand sides only when the groups still outnumber the
        // CTAs several times over: otherwise fewer, longer work units leave
        // the device idle at the end of the batch
        const bool group_rhs = systems >= 4 * kManyUnits;
        for (size_t q = 0; q < admit.size(); ++q) {
            ServerRequest& r = s->requests.at(admit[q]);
            const int n = s->patterns[r.pid].n;
            for (int c0 = 0; c0 < r.nrhs;) {
                const int rem = r.nrhs - c0;
                const int g = (group_rhs && rem >= 4) ? 4 : ((group_rhs && rem >= 2) ? 2 : 1);
                As.push_back(&sl.csrs[q]);
                Ms.push_back(r.F);
                bs.push_back(static_cast<const double*>(r.d_b) + (size_t)c0 * n);
                xs.push_back(static_cast<double*>(r.d_x) + (size_t)c0 * n);
                nrs.push_back(g);
                c0 += g;
            }
        }
        CULIPX_TRY(sqmr_solve_many_nr_async(sl.h, (int)As.size(), As.data(), Ms.data(), bs.data(), xs.data(),
                                            nrs.data(), s->tol, s->max_it, sl.h->sqmr, sl.out_host));
    }
    sl.reqs = admit;
    sl.busy = true;
    sl.large = large;
    ++s->batches;
    if (s->max_refine > 0) {
        // FP64 refinement: the true residuals of every right-hand side next
        sl.cols.clear();
        for (int id : admit)
            for (int c = 0; c < s->requests.at(id).nrhs; ++c) sl.cols.emplace_back(id, c);
        sl.phase = 1;
        return enqueue_residuals(s, sl, false);
    }
    sl.phase = 0;
    return enqueue_end(s, sl);
}

}  // namespace

int Server::running_slots() const
{
    int r = 0;
    for (const auto& sl : slots) r += sl.busy;
    return r;
}

long long ServerPattern::factor_bytes_estimate() const
{
    const Pattern& p = *pat;
    const long long vb = (precision == CULIPX_F64) ? 8 : 4;
    const long long slots = p.val_slots + 2 * p.sparse_slots;
    return slots * (vb + 4) * 2 + (long long)p.n * 64 + (long long)p.coarse_nnz * 24 + (long long)p.num_blocks * 64;
}

int server_progress(Server* s, int wait, int* completed)
{
    if (!s) return fail(CULIPX_INVALID_ARG, "null server");
    CULIPX_CUDA(cudaSetDevice(s->device));
    const long long done0 = s->done;
    for (;;) {
        // completions
        for (auto& sl : s->slots)
            if (sl.busy) {
                const cudaError_t e = cudaEventQuery(sl.done);
                if (e == cudaSuccess) {
                    CULIPX_TRY(launch_check("server batch"));
                    if (sl.phase == 1) {
                        CULIPX_TRY(refine_step(s, sl));  // a refinement round: corrections or the end
                        continue;
                    }
                    CULIPX_TRY(finish_slot(s, sl));
                } else if (e != cudaErrorNotReady) {
                    return fail(CULIPX_CUDA_ERROR, "server batch failed: %s", cudaGetErrorString(e));
                }
            }
        // admissions into free slots
        for (auto& sl : s->slots)
            if (!sl.busy && !s->queue.empty()) CULIPX_TRY(launch_slot(s, sl));
        if (!wait || s->done > done0 || s->running_slots() == 0) break;
        // block on the oldest busy slot
        for (auto& sl : s->slots)
            if (sl.busy) {
                CULIPX_CUDA(cudaEventSynchronize(sl.done));
                break;
            }
    }
    if (completed) *completed = (int)(s->done - done0);
    return CULIPX_OK;
}

int server_result(Server* s, int id, double* x, int* its, int* status, double* latency_ms)
{
    if (!s) return fail(CULIPX_INVALID_ARG, "null server");
    auto it = s->requests.find(id);
    if (it == s->requests.end()) return fail(CULIPX_INVALID_ARG, "culipx_server_result: unknown request %d", id);
    const ServerRequest& r = it->second;
    if (r.state != 2) return CULIPX_PENDING;
    if (x) std::memcpy(x, r.x.data(), r.x.size() * sizeof(double));
    if (its) std::memcpy(its, r.its.data(), r.its.size() * sizeof(int));
    if (status) std::memcpy(status, r.status.data(), r.status.size() * sizeof(int));
    if (latency_ms) *latency_ms = r.t_done - r.t_submit;
    return CULIPX_OK;
}

int server_release(Server* s, int id)
{
    if (!s) return fail(CULIPX_INVALID_ARG, "null server");
    auto it = s->requests.find(id);
    if (it == s->requests.end()) return fail(CULIPX_INVALID_ARG, "culipx_server_release: unknown request %d", id);
    if (it->second.state != 2) return fail(CULIPX_INVALID_ARG, "culipx_server_release: request %d not finished", id);
    s->requests.erase(it);
    return CULIPX_OK;
}

int server_stats(Server* s, long long* st8)
{
    if (!s || !st8) return fail(CULIPX_INVALID_ARG, "null argument");
    long long running = 0;
    for (const auto& sl : s->slots) running += (long long)sl.reqs.size();
    st8[0] = (long long)s->queue.size();
    st8[1] = running;
    st8[2] = s->done;
    st8[3] = s->batches;
    st8[4] = s->in_use;
    st8[5] = s->fixed_bytes();
    st8[6] = (long long)s->patterns.size();
    st8[7] = s->large_batches;
    return CULIPX_OK;
}

}  // namespace culipx
