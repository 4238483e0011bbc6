// Serving: continuous batching of band-solve requests on one GPU.
//
// A request is one cell at one k-point: its potential, plane-wave list,
// projectors, starting bands and Davidson options.  Requests queue in arrival
// order.  A worker thread picks the oldest request whose device-memory
// estimate fits the HBM budget beside the requests already running (one
// request is always admitted when nothing runs) and solves it in its own
// context, on its own stream.  Requests that arrive while others run start as
// soon as a worker and memory free up, and their kernels overlap with the
// others' on the device.  Each solve touches only its worker's buffers and
// every reduction in it has a fixed order, so a result does not depend on what
// else runs beside it.  Worker contexts keep their buffers between requests
// (no cudaFree, which would stall the other streams).
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "batcher.cuh"
#include "context.cuh"
#include "davidson.cuh"
#include "dense.cuh"
#include "q3b.h"

namespace q3b {
namespace {

template <typename V> void release(V& v) { V().swap(v); }

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Job {
    int id = 0;
    int n1 = 0, n2 = 0, n3 = 0;
    std::vector<double> v;
    int npw = 0, nproj = 0, natoms = 0, nb = 0;
    std::vector<int32_t> g2g, offs;
    std::vector<double> ke, dblk, eig;
    std::vector<double2> beta, bands;
    q3b_davidson_opts opts{};
    q3b_davidson_stats stats{};
    size_t est = 0;
    double t_submit = 0, t_start = 0, t_end = 0;
    int status = Q3B_OK;
    std::string err;
    bool done = false;
};

// device bytes a solve of this size holds (vectors, subspace matrices and the
// dense scratch, stick buffer, projectors, potential), with headroom
size_t estimate_bytes(const Job& j) {
    // the FP32 phase of a mixed solve holds a larger basis of 8-byte values, the
    // FP64 solve (and the mixed refinement) a basis of 16-byte values: the larger
    const bool mixed = j.opts.precision == Q3B_MIXED;
    const int factor = basis_factor(j.opts, j.nb, j.npw);
    const size_t nbi = mixed && factor > j.opts.basis_expansion_factor ? (size_t)mixed_bands(j.nb, j.npw)
                                                                       : (size_t)j.nb;  // buffer bands
    const size_t maxn = std::min<size_t>((size_t)std::max(2, factor) * nbi, j.npw);
    const size_t maxn64 = std::min<size_t>((size_t)std::max(2, j.opts.basis_expansion_factor) * nbi, j.npw);
    const size_t N = (size_t)j.n1 * j.n2 * j.n3;
    size_t b = 0;
    b += 3 * (size_t)j.npw * std::max(maxn * (mixed ? sizeof(float2) : sizeof(double2)), maxn64 * sizeof(double2));
    if (mixed) b += (size_t)j.npw * nbi * sizeof(double2);  // the bands between the two phases
    b += 10 * maxn * maxn * sizeof(double2) + dense::hegv_scratch_bytes((int)maxn) +
         dense::potrf_scratch_bytes((int)maxn);
    b += std::min<size_t>(48ull << 20, (size_t)j.nb * j.n3 * (size_t)j.n1 * j.n2 / 4 * sizeof(double2));
    // projectors: FP64, FP32 and the two packed tensor-core copies (16 B each)
    b += (size_t)j.npw * j.nproj * (sizeof(double2) + sizeof(float2) + 32);
    b += 2 * N * (sizeof(double) + sizeof(float));  // V/N in two layouts
    b += 2 * (size_t)j.nproj * j.nb * sizeof(double2) + (16ull << 20);
    return b + b / 5;
}

}  // namespace

class Server {
  public:
    Server(int device, size_t budget, int workers) : device_(device), budget_(budget) {
        if (workers < 1) workers = 1;
        for (int w = 0; w < workers; ++w) ctxs_.emplace_back(new q3b_context(device, 0));
        for (int w = 0; w < workers; ++w) threads_.emplace_back([this, w] { run(w); });
    }
    ~Server() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_work_.notify_all();
        for (auto& t : threads_) t.join();
    }

    int submit(std::unique_ptr<Job> j) {
        std::lock_guard<std::mutex> lk(mu_);
        j->id = next_id_++;
        j->t_submit = now_s();
        j->est = estimate_bytes(*j);
        Job* raw = j.get();
        jobs_[raw->id] = std::move(j);
        queue_.push_back(raw);
        cv_work_.notify_all();
        return raw->id;
    }

    Job* find(int id) {
        auto it = jobs_.find(id);
        return it == jobs_.end() ? nullptr : it->second.get();
    }

    // 1 done, 0 pending, -1 unknown id
    int poll(int id) {
        std::lock_guard<std::mutex> lk(mu_);
        Job* j = find(id);
        return j ? (j->done ? 1 : 0) : -1;
    }

    // Batch the workers' subspace eigensolves (batcher.cuh); only while no request is
    // queued or running.  wait_us: how long a batch waits for workers busy elsewhere.
    void set_batching(bool on, int wait_us) {
        std::lock_guard<std::mutex> lk(mu_);
        if (running_ > 0 || !queue_.empty())
            throw Status(Q3B_ERR_STATE, "batching can only change while the server is idle");
        batcher_.reset(on ? new EigenBatcher(device_, wait_us) : nullptr);
        for (auto& c : ctxs_) c->impl.batcher = batcher_.get();
    }
    void batch_stats(long* batches, long* problems) {
        std::lock_guard<std::mutex> lk(mu_);
        *batches = batcher_ ? batcher_->batches() : 0;
        *problems = batcher_ ? batcher_->problems() : 0;
    }

    std::unique_ptr<Job> wait(int id) {
        std::unique_lock<std::mutex> lk(mu_);
        Job* j = find(id);
        if (!j) return nullptr;
        cv_done_.wait(lk, [&] { return j->done; });
        auto it = jobs_.find(id);
        std::unique_ptr<Job> out = std::move(it->second);
        jobs_.erase(it);
        return out;
    }

    std::string err;

  private:
    void run(int w) {
        q3b_context* ctx = ctxs_[w].get();
        cudaSetDevice(device_);
        while (true) {
            Job* j = nullptr;
            EigenBatcher* batcher = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_work_.wait(lk, [&] {
                    if (stop_) return true;
                    return pick_locked() != queue_.end();
                });
                if (stop_) return;
                auto it = pick_locked();
                j = *it;
                queue_.erase(it);
                in_use_ += j->est;
                ++running_;
                batcher = batcher_.get();
                if (batcher) batcher->join();
            }
            j->t_start = now_s();
            solve(ctx, *j);
            j->t_end = now_s();
            if (batcher) batcher->leave();
            {
                std::lock_guard<std::mutex> lk(mu_);
                in_use_ -= j->est;
                --running_;
                j->done = true;
            }
            cv_done_.notify_all();
            cv_work_.notify_all();
        }
    }

    // oldest queued job that fits the budget beside the running ones
    std::deque<Job*>::iterator pick_locked() {
        for (auto it = queue_.begin(); it != queue_.end(); ++it) {
            if (running_ == 0 || budget_ == 0 || in_use_ + (*it)->est <= budget_) return it;
        }
        return queue_.end();
    }

    static void solve(q3b_context* ctx, Job& j) {
        Context& c = ctx->impl;
        try {
            Q3B_CUDA(cudaSetDevice(c.device));
            q3b::tc::ErrorScope scope(c.err_word.as<int>());
            c.set_potential(j.v.data(), j.n1, j.n2, j.n3);
            c.prepare_kpoint(j.npw, j.g2g.data(), j.ke.data(), j.nproj ? j.beta.data() : nullptr, j.nproj,
                             j.natoms, j.nproj ? j.offs.data() : nullptr, j.nproj ? j.dblk.data() : nullptr);
            // the inputs now live on the device: release their host copies, so that a
            // long stream holds host memory only for queued requests and results
            release(j.v);
            release(j.g2g);
            release(j.ke);
            release(j.beta);
            release(j.offs);
            release(j.dblk);
            const size_t bytes = (size_t)j.npw * j.nb * sizeof(double2);
            c.ws_bands.reserve(&c, bytes);
            Q3B_CUDA(cudaMemcpyAsync(c.ws_bands.ptr, j.bands.data(), bytes, cudaMemcpyHostToDevice, c.stream));
            davidson_solve(c, c.ws_bands.as<double2>(), j.eig.data(), j.nb, j.opts, &j.stats);
            Q3B_CUDA(cudaMemcpyAsync(j.bands.data(), c.ws_bands.ptr, bytes, cudaMemcpyDeviceToHost, c.stream));
            Q3B_CUDA(cudaStreamSynchronize(c.stream));
            j.status = Q3B_OK;
        } catch (const std::exception& e) {
            j.status = fail(ctx, e);
            j.err = e.what();
        }
    }

    int device_;
    size_t budget_;
    size_t in_use_ = 0;
    int running_ = 0;
    int next_id_ = 1;
    bool stop_ = false;
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    std::deque<Job*> queue_;
    std::map<int, std::unique_ptr<Job>> jobs_;
    std::unique_ptr<EigenBatcher> batcher_;
    std::vector<std::unique_ptr<q3b_context>> ctxs_;
    std::vector<std::thread> threads_;
};

}  // namespace q3b

struct q3b_server {
    std::unique_ptr<q3b::Server> impl;
    std::string err;
};

extern "C" {

int q3b_server_create(int device, size_t hbm_budget_bytes, int workers, q3b_server** out) {
    if (!out) return Q3B_ERR_INVALID;
    *out = nullptr;
    try {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
            cudaGetLastError();
            return Q3B_ERR_CUDA;
        }
        auto s = new q3b_server;
        s->impl.reset(new q3b::Server(device, hbm_budget_bytes, workers));
        *out = s;
        return Q3B_OK;
    } catch (const std::exception&) {
        return Q3B_ERR_CUDA;
    }
}

int q3b_server_set_batching(q3b_server* s, int enable, int wait_us) {
    if (!s) return Q3B_ERR_INVALID;
    try {
        s->impl->set_batching(enable != 0, wait_us > 0 ? wait_us : 200);
        return Q3B_OK;
    } catch (const q3b::Status& e) {
        s->err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        s->err = e.what();
        return Q3B_ERR_CUDA;
    }
}

int q3b_server_batch_stats(q3b_server* s, long* batches, long* problems) {
    if (!s || !batches || !problems) return Q3B_ERR_INVALID;
    s->impl->batch_stats(batches, problems);
    return Q3B_OK;
}

int q3b_server_destroy(q3b_server* s) {
    if (!s) return Q3B_ERR_INVALID;
    delete s;
    return Q3B_OK;
}

const char* q3b_server_last_error(const q3b_server* s) { return s ? s->err.c_str() : "null server"; }

int q3b_server_submit(q3b_server* s, const q3b_request* r, int* id_out) {
    if (!s || !r || !id_out) return Q3B_ERR_INVALID;
    try {
        if (r->n1 <= 0 || r->n2 <= 0 || r->n3 <= 0 || !r->v_r || r->npw <= 0 || !r->g_to_grid || !r->ke ||
            r->nb <= 0 || r->nb > r->npw || !r->bands || r->nproj < 0 ||
            (r->nproj > 0 && (!r->beta || r->natoms <= 0 || !r->atom_proj_offsets || !r->d_blocks))) {
            s->err = "q3b_server_submit: bad request";
            return Q3B_ERR_INVALID;
        }
        auto j = std::make_unique<q3b::Job>();
        const size_t N = (size_t)r->n1 * r->n2 * r->n3;
        j->n1 = r->n1;
        j->n2 = r->n2;
        j->n3 = r->n3;
        j->v.assign(r->v_r, r->v_r + N);
        j->npw = r->npw;
        j->nproj = r->nproj;
        j->natoms = r->natoms;
        j->nb = r->nb;
        j->g2g.assign(r->g_to_grid, r->g_to_grid + r->npw);
        j->ke.assign(r->ke, r->ke + r->npw);
        if (r->nproj > 0) {
            const auto* b = reinterpret_cast<const double2*>(r->beta);
            j->beta.assign(b, b + (size_t)r->npw * r->nproj);
            j->offs.assign(r->atom_proj_offsets, r->atom_proj_offsets + r->natoms + 1);
            size_t nd = 0;
            for (int a = 0; a < r->natoms; ++a) {
                const size_t m = (size_t)(r->atom_proj_offsets[a + 1] - r->atom_proj_offsets[a]);
                nd += m * m;
            }
            j->dblk.assign(r->d_blocks, r->d_blocks + nd);
        }
        const auto* b0 = reinterpret_cast<const double2*>(r->bands);
        j->bands.assign(b0, b0 + (size_t)r->npw * r->nb);
        j->eig.assign(r->nb, 0.0);
        if (r->eigenvalues) j->eig.assign(r->eigenvalues, r->eigenvalues + r->nb);
        if (r->opts) j->opts = *r->opts;
        else q3b_davidson_default_opts(&j->opts);
        j->opts.eigenvalue_history = nullptr;  // the caller's buffer is not written from a worker
        j->opts.history_rows = 0;
        *id_out = s->impl->submit(std::move(j));
        return Q3B_OK;
    } catch (const std::exception& e) {
        s->err = e.what();
        return Q3B_ERR_INTERNAL;
    }
}

int q3b_server_poll(q3b_server* s, int id) { return s ? s->impl->poll(id) : -1; }

int q3b_server_wait(q3b_server* s, int id, q3b_cplx128* bands_out, double* eig_out, q3b_davidson_stats* stats,
                    q3b_request_times* times) {
    if (!s) return Q3B_ERR_INVALID;
    auto j = s->impl->wait(id);
    if (!j) {
        s->err = "q3b_server_wait: unknown request id";
        return Q3B_ERR_INVALID;
    }
    if (bands_out) std::copy(j->bands.begin(), j->bands.end(), reinterpret_cast<double2*>(bands_out));
    if (eig_out) std::copy(j->eig.begin(), j->eig.end(), eig_out);
    if (stats) *stats = j->stats;
    if (times) {
        times->queue_ms = 1e3 * (j->t_start - j->t_submit);
        times->solve_ms = 1e3 * (j->t_end - j->t_start);
        times->latency_ms = 1e3 * (j->t_end - j->t_submit);
        times->estimated_bytes = j->est;
    }
    if (j->status != Q3B_OK) s->err = j->err;
    return j->status;
}

}  // extern "C"
