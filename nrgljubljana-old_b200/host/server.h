// NRG run server: many NRG runs in flight on one GPU (continuous batching).
//
// A request is one NRG run (a `param` + `data` work directory, results into
// an output directory).  Requests queue in arrival order; a free worker slot
// admits the head of the queue when its projected device memory fits in the
// budget next to the runs already admitted (a run always starts when nothing
// else runs).  The projection starts as an upper bound computed from the
// run's input and is then learned from the measured peaks of finished runs
// of the same shape; a run that runs out of memory on a learned projection
// is admitted once more on the bound.  Each worker drives its run with its own stream and host
// thread, so the GEMM, spectrum and binning work of different runs overlaps
// on the device.  The block eigensolves of all runs that are in their first
// sweep go through one batcher, which merges the blocks of the runs that
// are waiting into a single call of the batched solver: one set of
// cluster and panel launches then advance every run's blocks together.
// Runs that arrive while others are on the GPU join the next merged call.
//
// The reference has no counterpart: it runs one calculation per process
// (src/nrg.cc:3429-3469), parallelised inside a step over blocks
// (src/nrg.cc:2484-2507).
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../csrc/syev.cuh"
#include "driver.h"

namespace nrgb {

// Merges the eigensolver batches of concurrent runs (see above).  Requests
// fall in two classes: those whose blocks all fit the cluster
// tridiagonalisation, and those with larger blocks (which also need the
// cooperative panel launches).  Each class has its own queue and lanes; a
// lane is a thread with its own stream and solver.  The small class has
// NSMALL lanes, so a new merged call starts while the previous one still
// runs (these calls are latency-bound and leave most SMs free); the large
// class has one lane, so cooperative launches come from one lane only.
// Only one lane of a class gathers at a time.
class EigBatcher : public EigSolver {
 public:
  EigBatcher(int device, double window_us);
  ~EigBatcher() override;
  int solve(const std::vector<SyevDesc>& probs, cudaStream_t stream) override;
  void client_enter() override;
  void client_leave() override;
  // merged calls, requests served, problems solved
  void counters(double* calls, double* requests, double* problems);

 private:
  struct Req {
    const std::vector<SyevDesc>* probs = nullptr;
    cudaEvent_t ready = nullptr;
    bool done = false;
    int launches = 0;
    std::string err;
  };
  struct Lane {
    int cls = 0;  // 0: blocks that fit a cluster; 1: larger blocks
    std::unique_ptr<SyevBatched> syev;
    cudaStream_t stream = nullptr;
    int inflight = 0;  // requests in the lane's running merged call
    std::thread th;
  };
  static constexpr int NSMALL = 2;
  static constexpr int NLANE = NSMALL + 1;
  void loop(int lane);
  void run_batch(Lane& L, const std::vector<Req*>& batch);
  int pending_locked() const;

  int device_;
  double window_us_;
  int cluster_nmax_ = 0;  // blocks up to this size take the small class
  Lane lanes_[NLANE];
  std::deque<Req*> q_[2];              // queued requests per class
  bool gathering_[2] = {false, false};  // a lane of the class is gathering
  std::mutex m_;
  std::condition_variable cv_;       // a request arrived, a call ended, or stop
  std::condition_variable done_cv_;  // a merged call finished
  int clients_ = 0;  // runs inside their first sweep
  bool stop_ = false;
  long calls_ = 0, requests_ = 0, problems_ = 0;
};

// Upper bound of the device bytes one run holds at once, from its `param`
// and `data` (keep, Nmax, channels, tracked operators and spectra).
double project_run_bytes(const std::string& workdir);

// The bound and the shape of a run (keep, chain length, channels, tracked
// operators, density-matrix kind): runs of one shape hold similar memory.
struct RunShape {
  double bound = 0;
  std::string key;
};
RunShape run_shape(const std::string& workdir);

class Server {
 public:
  // mem_budget <= 0: 85% of the device memory free at creation.
  Server(int device, int max_runs, double mem_budget, double window_us);
  ~Server();  // finishes every queued and running request
  // Queue one run; returns its ticket (>= 1).  Throws if the input cannot be read.
  long long submit(const std::string& workdir, const std::string& outdir);
  // Wait for a ticket: 0 done, 2 failed (error text in *err), 7 timed out,
  // 1 unknown ticket.  stats[14]: the eight of nrgb_run, then latency
  // (submit to done), queue wait (submit to admission), projected bytes,
  // peak bytes held, eigensolver calls, admission order.
  int wait(long long ticket, double timeout_s, double* stats, std::string* err);
  // runs done, runs failed, merged eigensolver calls, requests, problems,
  // most runs in flight at once, most projected bytes admitted at once, budget
  void counters(double* out);

 private:
  using Clock = std::chrono::steady_clock;
  struct Job {
    long long id = 0;
    std::string wd, od;
    double bound = 0;       // upper bound of the run's device bytes
    std::string key;        // its shape (RunShape::key)
    double proj = 0;        // projection it was admitted with
    bool full_bound = false;  // admit on the bound (after running out of memory)
    Clock::time_point t_submit, t_admit, t_done;
    bool finished = false;
    int status = 0;
    std::string err;
    double st[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    RunExtra ex;
    long long order = 0;
  };
  void worker();
  // Admission projection: LEARN_MARGIN times the largest peak / bound ratio
  // measured for runs of the same shape, or twice that margin times the
  // largest ratio of any shape while none of this shape has finished, or
  // the bound while no run has finished (never above the bound).
  static constexpr double LEARN_MARGIN = 2.0;
  double projection(const Job& j) const;
  bool fits(const Job& j) const { return running_ == 0 || in_use_ + projection(j) <= budget_; }

  int device_;
  double budget_ = 0;
  EigBatcher batcher_;
  std::mutex m_;
  std::condition_variable work_cv_, done_cv_;
  std::deque<Job*> queue_;
  std::map<long long, std::unique_ptr<Job>> jobs_;
  long long next_id_ = 1, admitted_ = 0;
  double in_use_ = 0, peak_in_use_ = 0;
  int running_ = 0, peak_running_ = 0;
  std::map<std::string, double> ratio_;  // shape -> largest peak / bound seen
  long done_ = 0, failed_ = 0;
  bool stop_ = false;
  std::vector<std::thread> workers_;
};

}  // namespace nrgb
