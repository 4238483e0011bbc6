// Dynamic batching of the subspace eigensolves of concurrent Davidson solves.
//
// Solves that run at the same time on their own streams (the serving workers:
// different requests, or the k-points of one cell) each need one small
// generalized eigensolve per iteration.  Alone, each is a latency chain of a
// few dozen launches; here the solves that reach that step together share one
// launch of the one-block eigensolver (dense_block.cu), one block per problem.
//
// A solve hands its problem to EigenBatcher::solve and blocks.  The batch is
// launched by the thread whose arrival makes every running solve a member, or,
// after `wait_us` without that, by a waiting member: a solve that is busy
// elsewhere joins the next batch.  Ordering: each member's stream has recorded
// an event that the batch stream waits for before the launch, and each member's
// stream waits for the batch's completion event before its next kernel.  The
// eigenvalues come back to the host in the batch's one synchronisation.
//
// Which kernel solves a problem depends only on the problem (its order and
// vector count fit one block), never on the batch it lands in, and each block
// computes its problem independently: a solve's result is the same alone and
// in any mix.
#pragma once

#include <condition_variable>
#include <mutex>
#include <string>
#include <vector>

#include "dense.cuh"

namespace q3b {

class EigenBatcher {
  public:
    explicit EigenBatcher(int device, int wait_us = 200);
    ~EigenBatcher();
    EigenBatcher(const EigenBatcher&) = delete;
    EigenBatcher& operator=(const EigenBatcher&) = delete;

    // whether a problem goes through the batcher (it fits one block)
    static bool takes(int n, int nvec) { return dense::hegv_block_fits(n, nvec); }

    // Solve p (device pointers, as dense::hegv_block) after the work queued so
    // far on `st`; the nvec eigenvalues also to w_host.  Returns the problem's
    // status (0, or n + j as dense::hegv).  Blocks until done.
    int solve(const dense::BlockProblem& p, cudaStream_t st, double* w_host);

    // solves that are running and may submit (the batch waits for all of them)
    void join();
    void leave();

    // batches launched and problems solved (diagnostics)
    long batches() const { return batches_; }
    long problems() const { return problems_; }

  private:
    struct Ticket {
        dense::BlockProblem p;
        cudaEvent_t ready = nullptr;  // recorded on the member's stream at submission
        double* w_host = nullptr;
        int status = 0;
        bool done = false;
        int slot = 0;
    };
    void launch_locked(std::unique_lock<std::mutex>& lk);
    void run_batch(std::vector<Ticket*>& batch);

    int device_;
    int wait_us_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::vector<Ticket*> pending_;
    int members_ = 0;
    bool launching_ = false;
    long batches_ = 0, problems_ = 0;
    // batch resources (used by one launcher at a time)
    cudaStream_t stream_ = nullptr;
    cudaEvent_t finished_ = nullptr;
    std::vector<cudaEvent_t> free_events_;
    void* desc_dev_ = nullptr;    // BlockProblem[kMaxBatch]
    void* host_buf_ = nullptr;    // pinned: descriptors, then statuses and eigenvalues
    int* status_dev_ = nullptr;   // one status word per slot
    std::string err_;             // the last failed batch's message
    static constexpr int kMaxBatch = 64;
    static constexpr int kMaxOrder = 128;
};

}  // namespace q3b
