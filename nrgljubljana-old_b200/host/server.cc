// NRG run server (see server.h) and its C ABI (include/nrgb.h).
#include "server.h"

#include <math.h>
#include <string.h>

#include <algorithm>
#include <sstream>

#include "../../include/nrgb.h"
#include "data.h"
#include "params.h"

namespace nrgb {

// ---------------------------------------------------------------------------
// EigBatcher
// ---------------------------------------------------------------------------
EigBatcher::EigBatcher(int device, double window_us) : device_(device), window_us_(window_us) {
  NRGB_CUDA(cudaSetDevice(device_));
  for (int l = 0; l < NLANE; ++l) {
    lanes_[l].cls = l < NSMALL ? 0 : 1;
    lanes_[l].syev.reset(new SyevBatched());
    NRGB_CUDA(cudaStreamCreateWithFlags(&lanes_[l].stream, cudaStreamNonBlocking));
  }
  cluster_nmax_ = lanes_[0].syev->cluster_nmax();
  for (int l = 0; l < NLANE; ++l) lanes_[l].th = std::thread([this, l] { loop(l); });
}

EigBatcher::~EigBatcher() {
  {
    std::lock_guard<std::mutex> g(m_);
    stop_ = true;
  }
  cv_.notify_all();
  for (Lane& L : lanes_) {
    if (L.th.joinable()) L.th.join();
    L.syev.reset();
    if (L.stream) cudaStreamDestroy(L.stream);
  }
}

void EigBatcher::client_enter() {
  std::lock_guard<std::mutex> g(m_);
  ++clients_;
}

void EigBatcher::client_leave() {
  {
    std::lock_guard<std::mutex> g(m_);
    --clients_;
  }
  cv_.notify_all();  // a gathering call may now have every remaining client
}

void EigBatcher::counters(double* calls, double* requests, double* problems) {
  std::lock_guard<std::mutex> g(m_);
  *calls = (double)calls_;
  *requests = (double)requests_;
  *problems = (double)problems_;
}

int EigBatcher::pending_locked() const {
  int n = (int)q_[0].size() + (int)q_[1].size();
  for (const Lane& L : lanes_) n += L.inflight;
  return n;
}

int EigBatcher::solve(const std::vector<SyevDesc>& probs, cudaStream_t stream) {
  Req r;
  r.probs = &probs;
  int nmax = 0;
  for (const SyevDesc& d : probs) nmax = std::max(nmax, d.n);
  const int cls = (cluster_nmax_ > 0 && nmax <= cluster_nmax_) ? 0 : 1;
  NRGB_CUDA(cudaEventCreateWithFlags(&r.ready, cudaEventDisableTiming));
  NRGB_CUDA(cudaEventRecord(r.ready, stream));  // the blocks are assembled on the caller's stream
  {
    std::unique_lock<std::mutex> lk(m_);
    q_[cls].push_back(&r);
    cv_.notify_all();
    done_cv_.wait(lk, [&] { return r.done; });
  }
  cudaEventDestroy(r.ready);
  if (!r.err.empty()) throw CudaError(r.err);
  return r.launches;
}

void EigBatcher::loop(int lane) {
  cudaSetDevice(device_);
  Lane& L = lanes_[lane];
  const int k = L.cls;
  std::deque<Req*>& q = q_[k];
  std::unique_lock<std::mutex> lk(m_);
  for (;;) {
    cv_.wait(lk, [&] { return (stop_ && q.empty()) || (!q.empty() && !gathering_[k]); });
    if (q.empty()) return;  // stop requested and nothing pending in this class
    // gather: wait (at most the window) until every run inside its first
    // sweep has its blocks queued or being solved, in any lane
    gathering_[k] = true;
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::microseconds((long)window_us_);
    while (!stop_ && pending_locked() < clients_) {
      if (cv_.wait_until(lk, deadline) == std::cv_status::timeout) break;
    }
    gathering_[k] = false;
    std::vector<Req*> batch(q.begin(), q.end());
    q.clear();
    L.inflight = (int)batch.size();
    lk.unlock();
    run_batch(L, batch);
    lk.lock();
    L.inflight = 0;
    ++calls_;
    requests_ += (long)batch.size();
    for (Req* r : batch) {
      problems_ += (long)r->probs->size();
      r->done = true;
    }
    done_cv_.notify_all();
    cv_.notify_all();
  }
}

void EigBatcher::run_batch(Lane& L, const std::vector<Req*>& batch) {
  std::vector<SyevDesc> all;
  try {
    for (Req* r : batch) {
      NRGB_CUDA(cudaStreamWaitEvent(L.stream, r->ready, 0));
      all.insert(all.end(), r->probs->begin(), r->probs->end());
    }
    const int l = L.syev->solve(all, L.stream);
    for (Req* r : batch) r->launches = l;
    return;
  } catch (const std::exception& e) {
    cudaGetLastError();  // a launch error stays in this thread's last error until read
    if (batch.size() == 1) {
      batch[0]->err = e.what();
      return;
    }
  } catch (...) {
    // every request of the batch must be answered: its client waits for it
    cudaGetLastError();
    for (Req* r : batch) r->err = "eigensolver lane: unknown exception";
    return;
  }
  // a merged call failed: solve each run's blocks alone, so that only the
  // run whose blocks fail gets the error
  for (Req* r : batch) {
    try {
      r->launches = L.syev->solve(*r->probs, L.stream);
    } catch (const std::exception& e) {
      cudaGetLastError();
      r->err = e.what();
    } catch (...) {
      cudaGetLastError();
      r->err = "eigensolver lane: unknown exception";
    }
  }
}

// ---------------------------------------------------------------------------
// Memory projection
// ---------------------------------------------------------------------------
// K' = keep + safeguardmax bounds the multiplets kept after a step; every
// kept multiplet of the previous step enters at most `combs` blocks of the
// next one (combs = 4^channels), so D = combs K' bounds both the sum and the
// largest of the block dimensions, and D^2 bounds the eigenvector storage of
// a step.  The run keeps the eigenvectors of every step (the second sweep
// and the density matrices need them), one density matrix per step (two
// with FDM) of at most K'^2, and transients of a few D^2: the Hamiltonian,
// the recalculated operators and their intermediates.
double project_run_bytes(const std::string& wd) { return run_shape(wd).bound; }

RunShape run_shape(const std::string& wd) {
  Params P;
  P.read(wd + "/param");
  DataFile D;
  D.read(wd + "/data");
  const int Nmax = P.Nmax > 0 ? P.Nmax : D.Nmax;
  const double steps = std::max(1, Nmax - P.Ninit);
  const double kp = (double)P.keep + (P.safeguard > 0 ? (double)P.safeguardmax : 0.0);
  const double combs = pow(4.0, std::max(1, D.channels));
  const double dim = combs * kp;
  double nops = 0;
  for (const auto& k : D.ops) nops += (double)k.second.size();
  const double per_step = dim * dim + dim + (P.fdm ? 2.0 : 1.0) * kp * kp;
  const double transient = (3.0 + 2.0 * (nops + (double)D.channels)) * dim * dim;
  RunShape r;
  r.bound = 8.0 * (steps * per_step + transient) + 64.0 * (1 << 20);
  r.key = std::to_string(P.keep) + "/" + std::to_string(Nmax - P.Ninit) + "/" + std::to_string(D.channels) + "/" +
          std::to_string((int)nops) + (P.fdm ? "/fdm" : "") + (P.dmnrg ? "/dmnrg" : "");
  return r;
}

// ---------------------------------------------------------------------------
// Server
// ---------------------------------------------------------------------------
Server::Server(int device, int max_runs, double mem_budget, double window_us)
    : device_(device), batcher_(device, window_us) {
  NRGB_CUDA(cudaSetDevice(device));
  budget_ = mem_budget;
  if (budget_ <= 0) {
    size_t fr = 0, tot = 0;
    NRGB_CUDA(cudaMemGetInfo(&fr, &tot));
    budget_ = 0.85 * (double)fr;
  }
  max_runs = std::max(1, max_runs);
  for (int i = 0; i < max_runs; ++i) workers_.emplace_back([this] { worker(); });
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> g(m_);
    stop_ = true;
  }
  work_cv_.notify_all();
  for (auto& t : workers_)
    if (t.joinable()) t.join();
}

long long Server::submit(const std::string& wd, const std::string& od) {
  std::unique_ptr<Job> j(new Job);
  j->wd = wd;
  j->od = od;
  const RunShape shape = run_shape(wd);  // throws when the input cannot be read
  j->bound = shape.bound;
  j->key = shape.key;
  j->t_submit = Clock::now();
  std::lock_guard<std::mutex> g(m_);
  if (stop_) throw std::runtime_error("server is shutting down");
  j->id = next_id_++;
  const long long id = j->id;
  queue_.push_back(j.get());
  jobs_[id] = std::move(j);
  work_cv_.notify_all();
  return id;
}

void Server::worker() {
  cudaSetDevice(device_);
  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return;
  {
    NrgDriver drv(st, &batcher_);
    for (;;) {
      Job* j = nullptr;
      {
        std::unique_lock<std::mutex> lk(m_);
        // first come, first served: only the head of the queue is admitted
        work_cv_.wait(lk, [&] { return (stop_ && queue_.empty()) || (!queue_.empty() && fits(*queue_.front())); });
        if (queue_.empty()) break;
        j = queue_.front();
        queue_.pop_front();
        j->proj = projection(*j);
        in_use_ += j->proj;
        ++running_;
        peak_in_use_ = std::max(peak_in_use_, in_use_);
        peak_running_ = std::max(peak_running_, running_);
        j->order = ++admitted_;
        j->t_admit = Clock::now();
      }
      work_cv_.notify_all();  // the next head may fit too
      int status = 0;
      std::string err;
      try {
        drv.run(j->wd.c_str(), j->od.c_str(), j->st, &j->ex);
      } catch (const std::exception& e) {
        status = 2;
        err = e.what();
      }
      bool requeued = false;
      {
        std::lock_guard<std::mutex> g(m_);
        in_use_ -= j->proj;
        --running_;
        if (status == 0 && j->bound > 0) {
          double& r = ratio_[j->key];
          r = std::max(r, j->ex.peak_bytes / j->bound);
        }
        if (status != 0 && !j->full_bound && j->proj < j->bound &&
            err.find("out of memory") != std::string::npos) {
          // admitted on a learned projection and out of memory: once more,
          // at the head of the queue, on the full bound
          j->full_bound = true;
          queue_.push_front(j);
          requeued = true;
        } else {
          j->status = status;
          j->err = err;
          j->t_done = Clock::now();
          j->finished = true;
          if (status) ++failed_; else ++done_;
        }
      }
      if (requeued) {
        work_cv_.notify_all();
        continue;
      }
      done_cv_.notify_all();
      work_cv_.notify_all();
    }
  }
  cudaStreamDestroy(st);
}

double Server::projection(const Job& j) const {
  if (j.full_bound || ratio_.empty()) return j.bound;
  auto it = ratio_.find(j.key);
  if (it != ratio_.end()) return std::min(j.bound, LEARN_MARGIN * it->second * j.bound);
  // no run of this shape has finished yet: the largest ratio of any shape,
  // with a wider margin
  double r = 0;
  for (const auto& kv : ratio_) r = std::max(r, kv.second);
  return std::min(j.bound, 2.0 * LEARN_MARGIN * r * j.bound);
}

int Server::wait(long long ticket, double timeout_s, double* stats, std::string* err) {
  std::unique_lock<std::mutex> lk(m_);
  auto it = jobs_.find(ticket);
  if (it == jobs_.end()) return 1;
  Job* j = it->second.get();
  const auto pred = [&] { return j->finished; };
  if (timeout_s < 0) {
    done_cv_.wait(lk, pred);
  } else if (!done_cv_.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) {
    return 7;
  }
  if (stats) {
    for (int i = 0; i < 8; ++i) stats[i] = j->st[i];
    stats[8] = std::chrono::duration<double>(j->t_done - j->t_submit).count();
    stats[9] = std::chrono::duration<double>(j->t_admit - j->t_submit).count();
    stats[10] = j->proj;
    stats[11] = j->ex.peak_bytes;
    stats[12] = j->ex.eig_calls;
    stats[13] = (double)j->order;
  }
  if (err) *err = j->err;
  return j->status;
}

void Server::counters(double* out) {
  double calls = 0, reqs = 0, probs = 0;
  batcher_.counters(&calls, &reqs, &probs);
  std::lock_guard<std::mutex> g(m_);
  out[0] = (double)done_;
  out[1] = (double)failed_;
  out[2] = calls;
  out[3] = reqs;
  out[4] = probs;
  out[5] = (double)peak_running_;
  out[6] = peak_in_use_;
  out[7] = budget_;
}

}  // namespace nrgb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
struct nrgb_server {
  std::unique_ptr<nrgb::Server> s;
  std::mutex m;
  std::string err;                          // last error of a server call
  std::map<long long, std::string> run_err;  // error text per failed ticket
};

extern "C" {

int nrgb_server_create(int device, int max_runs, double mem_budget_bytes, double batch_window_us,
                       nrgb_server** out) {
  if (!out || max_runs < 1 || batch_window_us < 0) return 1;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return 3;
  if (device < 0 || device >= count) return 4;
  auto* h = new nrgb_server;
  try {
    h->s.reset(new nrgb::Server(device, max_runs, mem_budget_bytes, batch_window_us));
  } catch (const std::exception&) {
    delete h;
    return 2;
  }
  *out = h;
  return 0;
}

int nrgb_server_submit(nrgb_server* srv, const char* workdir, const char* outdir, long long* ticket) {
  if (!srv || !workdir || !outdir || !ticket) return 1;
  try {
    *ticket = srv->s->submit(workdir, outdir);
    return 0;
  } catch (const std::exception& e) {
    std::lock_guard<std::mutex> g(srv->m);
    srv->err = e.what();
    return 2;
  }
}

int nrgb_server_wait(nrgb_server* srv, long long ticket, double timeout_s, double* stats) {
  if (!srv) return 1;
  std::string err;
  const int rc = srv->s->wait(ticket, timeout_s, stats, &err);
  if (rc == 2) {
    std::lock_guard<std::mutex> g(srv->m);
    srv->run_err[ticket] = err;
    srv->err = err;
  }
  return rc;
}

const char* nrgb_server_error(nrgb_server* srv, long long ticket) {
  if (!srv) return "null server";
  std::lock_guard<std::mutex> g(srv->m);
  if (ticket <= 0) return srv->err.c_str();
  auto it = srv->run_err.find(ticket);
  return it == srv->run_err.end() ? "" : it->second.c_str();
}

int nrgb_server_counters(nrgb_server* srv, double* out) {
  if (!srv || !out) return 1;
  srv->s->counters(out);
  return 0;
}

int nrgb_server_destroy(nrgb_server* srv) {
  if (!srv) return 0;
  srv->s.reset();
  delete srv;
  return 0;
}

int nrgb_project_bytes(const char* workdir, double* bytes) {
  if (!workdir || !bytes) return 1;
  try {
    *bytes = nrgb::project_run_bytes(workdir);
    return 0;
  } catch (const std::exception&) {
    return 2;
  }
}

}  // extern "C"
