// serve.cu -- a decomposition server over the solvers of this library.
//
// No counterpart in the reference (cpd64 decomposes one tensor per run).
// Requests (a tensor in device COO form plus a CP-ALS or CP-APR job) are
// queued in arrival order and admitted against an HBM budget: a request
// starts when a worker is free and its estimated footprint fits in what the
// running requests leave.  Each worker owns a CUDA stream, so admitted
// requests run concurrently on the device.  A worker that admits a CP-ALS
// request also takes the CP-ALS requests queued behind it (same dtypes, up
// to max_batch, same iteration limit and tolerance, within the budget) and
// solves them together through the
// batched solver (batch.cu), so requests that arrive while others run join
// the next batch.  Each request's tensor is built on the worker's stream,
// its factors are initialised from the request's seed (the same values
// whether it runs alone or in a batch), and everything it allocated is
// freed when it completes.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "dense.cuh"

namespace altob {

// Uniform (0, 1) factor entries from a counter-based hash of (seed, mode,
// index): splitmix64 (Steele, Lea, Flood 2014), top 53 bits.
__device__ __forceinline__ double hash_uniform(u64 seed, u64 mode, u64 i)
{
    u64 z = seed * 0x9E3779B97F4A7C15ull + (mode << 48) + i + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return ((double)(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

template <typename FT>
__global__ void k_init_uniform(FT* __restrict__ U, u64 n, u64 seed, u64 mode)
{
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (u64)gridDim.x * blockDim.x)
        U[e] = (FT)hash_uniform(seed, mode, e);
}

template <typename FT>
__global__ void k_fill(FT* __restrict__ v, int n, FT x)
{
    for (int e = threadIdx.x; e < n; e += blockDim.x) v[e] = x;
}

static u64 footprint(const altob_request& r)
{
    const u64 vsz = r.vdtype == ALTOB_F64 ? 8 : 4;
    const u64 fsz = r.ftype == ALTOB_F64 ? 8 : 4;
    u64 rows = 0;
    for (int m = 0; m < r.nmode; ++m) rows += r.dims[m];
    const u64 build_peak = r.nnz * 48;                       // keys, payloads, ping-pong buffers
    const u64 resident = r.nnz * (8 + vsz + 4 * (u64)r.nmode);  // key, value, oidx
    const u64 model = rows * r.rank * fsz * (r.kind == ALTOB_REQ_CP_APR ? 4 : 2) +
                      r.dims[r.nmode - 1] * r.rank * fsz + (u64)r.nmode * r.rank * r.rank * 8 * 2;
    const bool apr = r.kind == ALTOB_REQ_CP_APR;
    const u64 pi = apr ? r.nnz * r.rank * fsz : 0;  // precomputed Khatri-Rao rows
    // row-ordered Phi stream (row, value, position per mode) and its sort scratch
    const u64 stream = apr ? r.nnz * ((u64)r.nmode * (8 + fsz) + 24) : 0;
    return std::max(build_peak, resident + pi + stream) + model + (16ull << 20);
}

struct Job {
    u64 id;
    altob_request req;
    altob_result res;
    u64 fp = 0;
    double est_s = 0.0;  // estimated device seconds (scheduling only)
    bool done = false;
};

// Work estimate of a request at an assumed 10 Gnnz/s of MTTKRP / Phi passes.
static double est_seconds(const altob_request& r)
{
    double passes = (double)r.nmode * (double)r.max_iters;
    if (r.kind == ALTOB_REQ_CP_APR) passes *= (double)std::max(1, r.max_inner);
    return (double)r.nnz * passes / 1e10;
}

}  // namespace altob

using namespace altob;

struct altob_server {
    altob_server_config cfg;
    std::chrono::steady_clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Job*> queue;
    std::map<u64, Job*> jobs;
    u64 next_id = 1;
    u64 used = 0, peak_used = 0;
    int running = 0;
    bool stop = false;
    std::vector<std::thread> workers;
    int device = 0;

    double now() const
    {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    // Next group to run, or empty: the first request by the policy (queue
    // order, or least estimated work net of waiting time) if it fits, plus
    // (CP-ALS) the queued CP-ALS requests that can share its batched solve.
    // Called with mu held.
    std::vector<Job*> take(int worker)
    {
        std::vector<Job*> g;
        if (queue.empty()) return g;
        auto pick = queue.begin();
        if (cfg.policy == 1) {
            const double t = now();
            double best = 1e300;
            for (auto it = queue.begin(); it != queue.end(); ++it) {
                const double score = (*it)->est_s - (t - (*it)->res.t_submit);
                if (score < best) {
                    best = score;
                    pick = it;
                }
            }
        }
        Job* h = *pick;
        if (h->fp > cfg.hbm_budget) {  // can never run
            queue.erase(pick);
            h->res.status = fail(ALTOB_ERR_NOMEM, "request footprint above the server's HBM budget");
            h->res.t_start = h->res.t_end = now();
            h->done = true;
            cv_done.notify_all();
            return take(worker);
        }
        if (used + h->fp > cfg.hbm_budget) return g;
        queue.erase(pick);
        used += h->fp;
        g.push_back(h);
        if (h->req.kind == ALTOB_REQ_CPD_ALS && !cfg.plain) {
            for (auto it = queue.begin(); it != queue.end() && (int)g.size() < cfg.max_batch;) {
                Job* j = *it;
                if (j->req.kind == ALTOB_REQ_CPD_ALS && j->req.ftype == h->req.ftype &&
                    j->req.vdtype == h->req.vdtype && j->req.max_iters == h->req.max_iters &&
                    j->req.tol == h->req.tol && used + j->fp <= cfg.hbm_budget) {
                    used += j->fp;
                    g.push_back(j);
                    it = queue.erase(it);
                } else {
                    ++it;
                }
            }
        }
        peak_used = std::max(peak_used, used);
        return g;
    }

    void worker_main(int worker)
    {
        cudaSetDevice(device);
        // batched CP-ALS solves (short, many small launches) run at the
        // device's highest stream priority, CP-APR requests (long streaming
        // passes) at the lowest, so a batch admitted while long requests
        // occupy the device still gets SMs as soon as blocks retire
        int lo = 0, hi = 0;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        cudaStream_t st = nullptr, st_hi = nullptr;
        cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, lo);
        cudaStreamCreateWithPriority(&st_hi, cudaStreamNonBlocking, cfg.plain ? lo : hi);
        for (;;) {
            std::vector<Job*> g;
            {
                std::unique_lock<std::mutex> lk(mu);
                for (;;) {
                    if (stop && queue.empty()) break;
                    g = take(worker);
                    if (!g.empty()) break;
                    cv_work.wait(lk);
                }
                if (g.empty()) break;
                ++running;
            }
            const double ts = now();
            for (Job* j : g) j->res.t_start = ts;
            run(g, g[0]->req.kind == ALTOB_REQ_CP_APR ? st : st_hi);
            {
                std::lock_guard<std::mutex> lk(mu);
                const double te = now();
                for (Job* j : g) {
                    used -= j->fp;
                    j->res.t_end = te;
                    j->res.batch_size = (int)g.size();
                    j->done = true;
                }
                --running;
            }
            cv_work.notify_all();
            cv_done.notify_all();
        }
        if (st) cudaStreamDestroy(st);
        if (st_hi) cudaStreamDestroy(st_hi);
    }

    struct Model {
        std::vector<void*> U;
        void* lam = nullptr;
    };

    altob_status alloc_model(const altob_request& r, cudaStream_t st, Model* m)
    {
        const size_t fsz = r.ftype == ALTOB_F64 ? 8 : 4;
        m->U.assign(r.nmode, nullptr);
        for (int k = 0; k < r.nmode; ++k) {
            ALTOB_CUDA(cudaMallocAsync(&m->U[k], r.dims[k] * r.rank * fsz, st));
            const u64 n = r.dims[k] * r.rank;
            const int grid = (int)std::min<u64>(1024, (n + 255) / 256);
            if (r.ftype == ALTOB_F64) k_init_uniform<double><<<grid, 256, 0, st>>>((double*)m->U[k], n, r.seed, k);
            else k_init_uniform<float><<<grid, 256, 0, st>>>((float*)m->U[k], n, r.seed, k);
        }
        ALTOB_CUDA(cudaMallocAsync(&m->lam, r.rank * fsz, st));
        if (r.ftype == ALTOB_F64) k_fill<double><<<1, 128, 0, st>>>((double*)m->lam, (int)r.rank, 1.0);
        else k_fill<float><<<1, 128, 0, st>>>((float*)m->lam, (int)r.rank, 1.0f);
        ALTOB_LAUNCH_CHECK();
        return ALTOB_OK;
    }

    static void free_model(Model& m, cudaStream_t st)
    {
        for (void* p : m.U)
            if (p) cudaFreeAsync(p, st);
        if (m.lam) cudaFreeAsync(m.lam, st);
        m.U.clear();
        m.lam = nullptr;
    }

    void run(std::vector<Job*>& g, cudaStream_t st)
    {
        const int n = (int)g.size();
        std::vector<altob_tensor*> ts(n, nullptr);
        std::vector<Model> ms(n);
        altob_status s = ALTOB_OK;
        for (int b = 0; b < n && s == ALTOB_OK; ++b) {
            const altob_request& r = g[b]->req;
            s = altob_create_device(r.nmode, r.dims, r.nnz, (const uint64_t*)r.d_cidx, r.d_vals, r.vdtype,
                                    r.nprtn > 0 ? r.nprtn : 128, 0, st, &ts[b]);
            if (s == ALTOB_OK) s = alloc_model(r, st, &ms[b]);
        }
        if (s == ALTOB_OK) {
            const altob_request& r0 = g[0]->req;
            if (r0.kind == ALTOB_REQ_CP_APR) {
                double out[5] = {0, 0, 0, 0, 0};
                s = altob_cp_apr(ts[0], r0.ftype, ms[0].U.data(), ms[0].lam, r0.rank, r0.max_iters, r0.max_inner,
                                 r0.tol, 1e-10, 1e-10, 1e-2, 0, out, st);
                g[0]->res.loglik = out[0];
                g[0]->res.fit = out[1];
                g[0]->res.iters = (int)out[3];
            } else if (cfg.plain) {
                std::vector<double> fits(r0.max_iters, 0.0);
                int it = 0;
                s = altob_cpd_als(ts[0], r0.ftype, ms[0].U.data(), ms[0].lam, r0.rank, r0.max_iters, r0.tol,
                                  fits.data(), &it, st);
                g[0]->res.iters = it;
                g[0]->res.fit = it > 0 ? fits[it - 1] : 0.0;
            } else {
                std::vector<uint64_t> ranks(n);
                std::vector<void* const*> fac(n);
                std::vector<void*> lam(n);
                for (int b = 0; b < n; ++b) {
                    ranks[b] = g[b]->req.rank;
                    fac[b] = ms[b].U.data();
                    lam[b] = ms[b].lam;
                }
                // one batched solve runs one iteration limit and tolerance:
                // only requests that share them are batched (take())
                const int iters_max = r0.max_iters;
                altob_batch* bh = nullptr;
                s = altob_batch_create(ts.data(), n, ranks.data(), r0.ftype, fac.data(), lam.data(), iters_max, st,
                                       &bh);
                if (s == ALTOB_OK && cfg.autotune) s = altob_batch_autotune(bh, 0, st);
                std::vector<double> fits((size_t)n * iters_max, 0.0);
                std::vector<int> its(n, 0);
                if (s == ALTOB_OK)
                    s = altob_batch_cpd_als(bh, iters_max, r0.tol, fits.data(), its.data(), cfg.use_graph, st);
                altob_batch_destroy(bh);
                for (int b = 0; b < n; ++b) {
                    g[b]->res.iters = its[b];
                    g[b]->res.fit = its[b] > 0 ? fits[(size_t)b * iters_max + its[b] - 1] : 0.0;
                }
            }
        }
        cudaStreamSynchronize(st);  // the solvers return with their work done; builds may have failed midway
        for (int b = 0; b < n; ++b) {
            if (ts[b]) altob_destroy(ts[b]);
            free_model(ms[b], st);
        }
        cudaStreamSynchronize(st);
        for (Job* j : g) j->res.status = s;
    }
};

extern "C" {

altob_status altob_request_footprint(const altob_request* r, uint64_t* bytes)
{
    if (!r || !bytes) return fail(ALTOB_ERR_ARG, "NULL argument");
    if (r->nmode < 2 || r->nmode > ALTOB_MAX_MODES) return fail(ALTOB_ERR_ARG, "nmode out of range");
    *bytes = footprint(*r);
    return ALTOB_OK;
}

altob_status altob_server_create(const altob_server_config* cfg, altob_server** out)
{
    if (!cfg || !out) return fail(ALTOB_ERR_ARG, "NULL argument");
    *out = nullptr;
    if (cfg->workers < 1 || cfg->workers > 64) return fail(ALTOB_ERR_ARG, "workers must be 1..64");
    if (cfg->max_batch < 1) return fail(ALTOB_ERR_ARG, "max_batch must be >= 1");
    if (cfg->hbm_budget == 0) return fail(ALTOB_ERR_ARG, "HBM budget must be > 0");
    if (cfg->policy != 0 && cfg->policy != 1) return fail(ALTOB_ERR_ARG, "policy must be 0 or 1");
    int dev = 0;
    ALTOB_CUDA(cudaGetDevice(&dev));
    altob_server* s = new altob_server();
    s->cfg = *cfg;
    s->device = dev;
    s->t0 = std::chrono::steady_clock::now();
    for (int w = 0; w < cfg->workers; ++w) s->workers.emplace_back([s, w] { s->worker_main(w); });
    *out = s;
    return ALTOB_OK;
}

double altob_server_clock(const altob_server* s) { return s ? s->now() : 0.0; }

altob_status altob_server_submit(altob_server* s, const altob_request* r, uint64_t* id)
{
    if (!s || !r || !id) return fail(ALTOB_ERR_ARG, "NULL argument");
    if (r->nmode < 2 || r->nmode > ALTOB_MAX_MODES) return fail(ALTOB_ERR_ARG, "nmode out of range");
    if (r->kind != ALTOB_REQ_CPD_ALS && r->kind != ALTOB_REQ_CP_APR) return fail(ALTOB_ERR_ARG, "unknown kind");
    if (r->nnz == 0 || !r->d_cidx || !r->d_vals) return fail(ALTOB_ERR_ARG, "empty request");
    if (r->rank < 1 || r->rank > (u64)SOLVE_MAX_RANK) return fail(ALTOB_ERR_UNSUPPORTED, "rank must be 1..112");
    if (r->max_iters < 1) return fail(ALTOB_ERR_ARG, "max_iters must be >= 1");
    Job* j = new Job();
    j->req = *r;
    memset(&j->res, 0, sizeof(j->res));
    j->fp = footprint(*r);
    j->est_s = est_seconds(*r);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            delete j;
            return fail(ALTOB_ERR_ARG, "server is shutting down");
        }
        j->id = s->next_id++;
        j->res.t_submit = s->now();
        s->jobs[j->id] = j;
        s->queue.push_back(j);
        *id = j->id;
    }
    s->cv_work.notify_one();
    return ALTOB_OK;
}

altob_status altob_server_wait(altob_server* s, uint64_t id, altob_result* out)
{
    if (!s || !out) return fail(ALTOB_ERR_ARG, "NULL argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return fail(ALTOB_ERR_ARG, "unknown request id");
    Job* j = it->second;
    s->cv_done.wait(lk, [j] { return j->done; });
    *out = j->res;
    s->jobs.erase(it);
    delete j;
    return ALTOB_OK;
}

altob_status altob_server_stats(const altob_server* s, uint64_t* used, uint64_t* peak, int* queued, int* running)
{
    if (!s) return fail(ALTOB_ERR_ARG, "NULL server");
    altob_server* m = const_cast<altob_server*>(s);
    std::lock_guard<std::mutex> lk(m->mu);
    if (used) *used = m->used;
    if (peak) *peak = m->peak_used;
    if (queued) *queued = (int)m->queue.size();
    if (running) *running = m->running;
    return ALTOB_OK;
}

altob_status altob_server_destroy(altob_server* s)
{
    if (!s) return ALTOB_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) t.join();
    for (auto& kv : s->jobs) delete kv.second;
    delete s;
    return ALTOB_OK;
}

}  // extern "C"
