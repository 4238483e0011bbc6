// EigenBatcher: the subspace eigensolves of concurrent solves in shared
// launches (batcher.cuh).
#include <algorithm>
#include <chrono>
#include <cstring>

#include "batcher.cuh"
#include "context.cuh"
#include "q3b.h"

namespace q3b {

EigenBatcher::EigenBatcher(int device, int wait_us) : device_(device), wait_us_(std::max(1, wait_us)) {
    Q3B_CUDA(cudaSetDevice(device_));
    Q3B_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    Q3B_CUDA(cudaEventCreateWithFlags(&finished_, cudaEventDisableTiming));
    Q3B_CUDA(cudaMalloc(&desc_dev_, kMaxBatch * sizeof(dense::BlockProblem)));
    Q3B_CUDA(cudaMalloc(reinterpret_cast<void**>(&status_dev_), kMaxBatch * sizeof(int)));
    Q3B_CUDA(cudaMallocHost(&host_buf_, kMaxBatch * sizeof(dense::BlockProblem) + kMaxBatch * sizeof(int) +
                                            (size_t)kMaxBatch * kMaxOrder * sizeof(double)));
}

EigenBatcher::~EigenBatcher() {
    cudaSetDevice(device_);
    if (stream_) cudaStreamSynchronize(stream_);
    for (cudaEvent_t e : free_events_) cudaEventDestroy(e);
    if (finished_) cudaEventDestroy(finished_);
    if (desc_dev_) cudaFree(desc_dev_);
    if (status_dev_) cudaFree(status_dev_);
    if (host_buf_) cudaFreeHost(host_buf_);
    if (stream_) cudaStreamDestroy(stream_);
}

void EigenBatcher::join() {
    std::lock_guard<std::mutex> lk(mu_);
    ++members_;
}

void EigenBatcher::leave() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        --members_;
    }
    cv_.notify_all();  // the batch may now hold every remaining member
}

int EigenBatcher::solve(const dense::BlockProblem& p, cudaStream_t st, double* w_host) {
    if (!takes(p.n, p.nvec) || p.nvec > kMaxOrder)
        throw Status(Q3B_ERR_INVALID, "eigensolve batch: problem does not fit one block");
    Ticket t;
    t.p = p;
    t.w_host = w_host;
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (!free_events_.empty()) {
            t.ready = free_events_.back();
            free_events_.pop_back();
        }
    }
    if (!t.ready) Q3B_CUDA(cudaEventCreateWithFlags(&t.ready, cudaEventDisableTiming));
    Q3B_CUDA(cudaEventRecord(t.ready, st));
    std::unique_lock<std::mutex> lk(mu_);
    pending_.push_back(&t);
    while (!t.done) {
        if (!launching_ && !pending_.empty() && (int)pending_.size() >= members_) {
            launch_locked(lk);
            continue;
        }
        const auto r = cv_.wait_for(lk, std::chrono::microseconds(wait_us_));
        if (r == std::cv_status::timeout && !t.done && !launching_ && !pending_.empty()) launch_locked(lk);
    }
    free_events_.push_back(t.ready);
    const int status = t.status;
    const std::string err = err_;
    lk.unlock();
    if (status == -1) throw Status(Q3B_ERR_CUDA, "eigensolve batch failed: " + err);
    return status;
}

// mu_ held on entry and on return; released while the batch runs
void EigenBatcher::launch_locked(std::unique_lock<std::mutex>& lk) {
    launching_ = true;
    const size_t take = std::min<size_t>(pending_.size(), kMaxBatch);
    std::vector<Ticket*> batch(pending_.begin(), pending_.begin() + take);
    pending_.erase(pending_.begin(), pending_.begin() + take);
    lk.unlock();
    bool ok = true;
    std::string what;
    try {
        run_batch(batch);
    } catch (const std::exception& e) {
        ok = false;
        what = e.what();
    }
    lk.lock();
    if (!ok) err_ = what;
    for (Ticket* t : batch) {
        if (!ok) t->status = -1;
        t->done = true;
    }
    ++batches_;
    problems_ += (long)batch.size();
    launching_ = false;
    cv_.notify_all();
}

void EigenBatcher::run_batch(std::vector<Ticket*>& batch) {
    Q3B_CUDA(cudaSetDevice(device_));
    const int count = static_cast<int>(batch.size());
    auto* desc = static_cast<dense::BlockProblem*>(host_buf_);
    int* status = reinterpret_cast<int*>(desc + kMaxBatch);
    double* wst = reinterpret_cast<double*>(status + kMaxBatch);
    size_t smem = 0;
    for (int i = 0; i < count; ++i) {
        Ticket* t = batch[i];
        Q3B_CUDA(cudaStreamWaitEvent(stream_, t->ready, 0));
        desc[i] = t->p;
        desc[i].info = status_dev_ + i;
        smem = std::max(smem, dense::hegv_block_smem(t->p.n, t->p.nvec));
    }
    Q3B_CUDA(cudaMemcpyAsync(desc_dev_, desc, count * sizeof(dense::BlockProblem), cudaMemcpyHostToDevice,
                             stream_));
    dense::hegv_block_many(stream_, static_cast<const dense::BlockProblem*>(desc_dev_), count, smem);
    Q3B_CUDA(cudaMemcpyAsync(status, status_dev_, count * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    for (int i = 0; i < count; ++i) {
        Ticket* t = batch[i];
        if (t->w_host)
            Q3B_CUDA(cudaMemcpyAsync(wst + (size_t)i * kMaxOrder, t->p.w, t->p.nvec * sizeof(double),
                                     cudaMemcpyDeviceToHost, stream_));
    }
    Q3B_CUDA(cudaEventRecord(finished_, stream_));
    Q3B_CUDA(cudaEventSynchronize(finished_));
    for (int i = 0; i < count; ++i) {
        Ticket* t = batch[i];
        t->status = status[i];
        if (t->w_host) std::memcpy(t->w_host, wst + (size_t)i * kMaxOrder, t->p.nvec * sizeof(double));
    }
}

}  // namespace q3b
