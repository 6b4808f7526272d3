// KernelStats (common.cuh): launch counters and event timing per kernel name.
#include <string.h>

#include "common.cuh"

namespace nrgb {

KernelStats& KernelStats::get() {
  static KernelStats s;
  return s;
}

cudaEvent_t KernelStats::ev() {
  if (!pool_.empty()) {
    cudaEvent_t e = pool_.back();
    pool_.pop_back();
    return e;
  }
  cudaEvent_t e;
  NRGB_CUDA(cudaEventCreate(&e));
  return e;
}

namespace {
// `name` matches `pat`: "*" (everything), a prefix ending in '*', or the
// name itself
bool name_matches(const char* name, const char* pat) {
  const size_t len = strlen(pat);
  if (len == 1 && pat[0] == '*') return true;
  if (len > 1 && pat[len - 1] == '*') return strncmp(name, pat, len - 1) == 0;
  return strcmp(name, pat) == 0;
}
}  // namespace

void KernelStats::enable(bool on, const char* only) {
  std::lock_guard<std::mutex> g(m_);
  settle();
  counts_.clear();
  ms_.clear();
  work_.clear();
  timing_ = on;
  only_ = only ? only : "";
}

int KernelStats::begin(const char* name, cudaStream_t s) {
  std::lock_guard<std::mutex> g(m_);
  count_locked(name, 1);
  if (!timing_ || (!only_.empty() && !name_matches(name, only_.c_str()))) return -1;
  int slot;
  if (!free_.empty()) {
    slot = free_.back();
    free_.pop_back();
  } else {
    slot = (int)open_.size();
    open_.push_back(Rec{});
  }
  open_[slot] = Rec{name, ev(), ev()};
  NRGB_CUDA(cudaEventRecord(open_[slot].a, s));
  return slot;
}

void KernelStats::end(int slot, cudaStream_t s) {
  if (slot < 0) return;
  std::lock_guard<std::mutex> g(m_);
  if (slot >= (int)open_.size()) return;
  Rec r = open_[slot];
  free_.push_back(slot);
  NRGB_CUDA(cudaEventRecord(r.b, s));
  done_.push_back(r);
  if (done_.size() > 4096) settle();
}

void KernelStats::count(const char* name, long n) {
  std::lock_guard<std::mutex> g(m_);
  count_locked(name, n);
}

void KernelStats::add_work(const char* name, double units) {
  std::lock_guard<std::mutex> g(m_);
  for (auto& w : work_)
    if (w.first == name) {
      w.second += units;
      return;
    }
  work_.push_back({name, units});
}

double KernelStats::work(const char* name) {
  std::lock_guard<std::mutex> g(m_);
  const bool all = strcmp(name, "*") == 0;
  const size_t len = strlen(name);
  const bool prefix = len > 1 && name[len - 1] == '*';
  double t = 0;
  for (auto& w : work_) {
    const std::string& k = w.first;
    if (all || (prefix ? k.compare(0, len - 1, name, len - 1) == 0 : k == name)) t += w.second;
  }
  return t;
}

void KernelStats::count_locked(const char* name, long n) {
  for (auto& c : counts_)
    if (c.first == name) {
      c.second += n;
      return;
    }
  counts_.push_back({name, n});
}

void KernelStats::settle() {
  // Take the finished records out of done_ first: each record is counted at
  // most once and its events go back to the pool exactly once, even when a
  // CUDA error ends the loop early (the failed record and the ones after it
  // are dropped, and the error is reported once at the end).
  std::vector<Rec> recs;
  recs.swap(done_);
  cudaError_t first_err = cudaSuccess;
  for (const Rec& r : recs) {
    float ms = 0.f;
    cudaError_t e = first_err == cudaSuccess ? cudaEventSynchronize(r.b) : first_err;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, r.a, r.b);
    if (e == cudaSuccess) {
      bool found = false;
      for (auto& m : ms_)
        if (m.first == r.name) {
          m.second += ms;
          found = true;
        }
      if (!found) ms_.push_back({r.name, (double)ms});
    } else if (first_err == cudaSuccess) {
      first_err = e;
    }
    pool_.push_back(r.a);
    pool_.push_back(r.b);
  }
  NRGB_CUDA(first_err);
}

void KernelStats::query(const char* name, long* launches, double* ms) {
  std::lock_guard<std::mutex> g(m_);
  settle();
  const bool all = strcmp(name, "*") == 0;
  const size_t len = strlen(name);
  const bool prefix = len > 1 && name[len - 1] == '*';
  auto match = [&](const std::string& k) {
    if (all) return true;
    if (prefix) return k.compare(0, len - 1, name, len - 1) == 0;
    return k == name;
  };
  long n = 0;
  double t = 0;
  for (auto& c : counts_)
    if (match(c.first)) n += c.second;
  for (auto& m : ms_)
    if (match(m.first)) t += m.second;
  if (launches) *launches = n;
  if (ms) *ms = t;
}

}  // namespace nrgb
