// Serving scheduler (see serve.hpp).  Host code only: every proof runs through
// Setup::prove on the setup's own stream.
#include "serve.hpp"
#include "../../include/flock_gpu.h"
#include <atomic>

namespace flock {

Server::Server(int device, uint64_t budget, int slots) : device_(device), budget_(budget) {
  if (slots < 1 || slots > 64) throw std::runtime_error("serving slots must be in 1..64");
  n_slots_ = slots;
  for (int i = 0; i < slots; i++) {
    const bool small_only = slots >= 3 && i < std::max(1, slots / 4);  // the express slots
    workers_.emplace_back([this, small_only] { worker(small_only); });
  }
}

// One proof's device time: about 6 M compressions per second plus a fixed
// per-proof cost (host round trips, launches) of about 1 ms.
double Server::expected_ms(uint32_t log2) { return 1.0 + (double)(1u << log2) / 6.0e3; }

size_t Server::pick(bool small_only) const {
  const auto now = Clock::now();
  size_t best = queue_.size();
  double best_score = 0;
  for (size_t i = 0; i < queue_.size(); i++) {
    const Job& j = queue_[i];
    if (small_only && j.log2 > kSmallLog2) continue;
    const double waited = std::chrono::duration<double, std::milli>(now - j.submitted).count();
    const double score = expected_ms(j.log2) - waited / kAging;
    if (best == queue_.size() || score < best_score) {
      best = i;
      best_score = score;
    }
  }
  return best;
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  cv_jobs_.notify_all();
  cv_mem_.notify_all();
  for (auto& t : workers_) t.join();
  std::lock_guard<std::mutex> bl(batch_mu_);
  idle_.clear();  // frees the cached setups
  if (batch_st_) cudaStreamDestroy(batch_st_);
}

void Server::self_check(Setup& s, const std::string& domain, JobResult& r) {
  if (!verify_) return;
  const std::string why = s.verify(r.bytes.data(), r.bytes.size(), domain);
  if (!why.empty()) {
    r.status = FLOCK_ERR_VERIFY;
    r.error = "self-check failed: " + why;
  }
}

std::vector<JobResult> Server::prove_batch(const std::vector<BatchItem>& jobs, int threads) {
  std::lock_guard<std::mutex> bl(batch_mu_);
  cudaSetDevice(device_);
  if (!batch_st_) CK(cudaStreamCreateWithFlags(&batch_st_, cudaStreamNonBlocking));
  if (threads < 1) threads = 1;
  auto ms = [](Clock::duration d) { return std::chrono::duration<double, std::milli>(d).count(); };
  const auto t0 = Clock::now();
  std::vector<JobResult> res(jobs.size());
  size_t next = 0;
  while (next < jobs.size()) {
    // admit a wave: as many jobs, in order, as fit the budget now
    std::vector<std::pair<size_t, std::unique_ptr<Setup>>> wave;
    {
      std::unique_lock<std::mutex> lk(mu_);
      while (next < jobs.size()) {
        std::unique_ptr<Setup> s;
        try {
          s = acquire(jobs[next].log2, lk, wave.empty());
        } catch (const std::exception& e) {
          res[next].status = FLOCK_ERR_CAPACITY;
          res[next].error = e.what();
          next++;
          continue;
        }
        if (!s) break;
        wave.emplace_back(next++, std::move(s));
      }
    }
    if (wave.empty()) continue;
    const auto t_run = Clock::now();
    // The seeded jobs' fused commits are queued in groups, in order, on the
    // batch stream; a job's remaining phases start (on its own stream, after
    // its group's commit) as soon as its group is queued, so the commit of
    // one group overlaps the transcript phases of the earlier ones.
    constexpr size_t kGroup = 8;
    const size_t nw = wave.size();
    std::unique_ptr<std::atomic<int>[]> ready(new std::atomic<int>[nw]);  // 0 wait, 1 go, 2 commit failed
    std::vector<std::string> commit_err(nw);
    std::vector<size_t> seeded;
    for (size_t i = 0; i < nw; i++) {
      const bool blocks = jobs[wave[i].first].blocks != nullptr;
      ready[i].store(blocks ? 1 : 0);
      if (!blocks) seeded.push_back(i);
    }
    std::mutex rmu;
    std::condition_variable rcv;
    std::atomic<size_t> k{0};
    auto run = [&] {
      cudaSetDevice(device_);
      for (size_t i; (i = k.fetch_add(1)) < nw;) {
        {
          std::unique_lock<std::mutex> rl(rmu);
          rcv.wait(rl, [&] { return ready[i].load() != 0; });
        }
        const BatchItem& job = jobs[wave[i].first];
        Setup& S = *wave[i].second;
        S.grid_sms = 0;  // a batch keeps every SM busy
        JobResult& r = res[wave[i].first];
        try {
          if (ready[i].load() == 2) throw std::runtime_error("batch commit: " + commit_err[i]);
          if (job.blocks) {
            const size_t n = (size_t)1 << job.log2;
            if (!S.blocks_buf)
              CK(cudaMallocAsync(reinterpret_cast<void**>(&S.blocks_buf), n * 25 * sizeof(uint32_t), S.st));
            CK(cudaMemcpyAsync(S.blocks_buf, job.blocks, n * 25 * sizeof(uint32_t), cudaMemcpyHostToDevice, S.st));
            r.bytes = S.prove(nullptr, S.blocks_buf, n, job.domain);
          } else {
            r.bytes = S.prove(&job.seed, nullptr, 0, job.domain, true);
          }
          r.status = FLOCK_OK;
          self_check(S, job.domain, r);
        } catch (const CudaError& e) {
          r.status = FLOCK_ERR_CUDA;
          r.error = e.what();
        } catch (const std::exception& e) {
          r.status = FLOCK_ERR_INTERNAL;
          r.error = e.what();
        }
        const auto t_end = Clock::now();
        r.queue_ms = ms(t_run - t0);
        r.run_ms = ms(t_end - t_run);
        r.latency_ms = ms(t_end - t0);
      }
    };
    std::vector<std::thread> th;
    for (int t = 0; t < threads && t < (int)nw; t++) th.emplace_back(run);
    std::vector<BatchCommit> handles;
    for (size_t g0 = 0; g0 < seeded.size(); g0 += kGroup) {
      const size_t g1 = std::min(seeded.size(), g0 + kGroup);
      std::vector<Setup*> ss;
      std::vector<uint64_t> seeds;
      for (size_t j = g0; j < g1; j++) {
        ss.push_back(wave[seeded[j]].second.get());
        seeds.push_back(jobs[wave[seeded[j]].first].seed);
      }
      int state = 1;
      try {
        handles.push_back(batch_commit_async(ss, seeds, batch_st_));
      } catch (const std::exception& e) {
        state = 2;
        for (size_t j = g0; j < g1; j++) commit_err[seeded[j]] = e.what();
      }
      {
        std::lock_guard<std::mutex> rl(rmu);
        for (size_t j = g0; j < g1; j++) ready[seeded[j]].store(state);
      }
      rcv.notify_all();
    }
    for (auto& t : th) t.join();
    cudaStreamSynchronize(batch_st_);
    for (auto& h : handles) batch_commit_release(h);
    std::lock_guard<std::mutex> lk(mu_);
    for (auto& w : wave) release(std::move(w.second));
  }
  return res;
}

uint64_t Server::submit(uint32_t log2, uint64_t seed, const uint32_t* blocks, const std::string& domain) {
  Job j;
  j.log2 = log2;
  j.seed = seed;
  j.domain = domain;
  if (blocks) {
    j.has_blocks = true;
    j.blocks.assign(blocks, blocks + ((size_t)25 << log2));
  }
  j.submitted = Clock::now();
  uint64_t t;
  {
    std::lock_guard<std::mutex> lk(mu_);
    if (stop_) throw std::runtime_error("server stopped");
    t = j.ticket = next_ticket_++;
    queue_.push_back(std::move(j));
  }
  cv_jobs_.notify_all();  // the express slot takes only small jobs: wake every slot
  return t;
}

bool Server::wait(uint64_t ticket, int timeout_ms, JobResult* out) {
  std::unique_lock<std::mutex> lk(mu_);
  auto ready = [&] { return done_.count(ticket) > 0; };
  if (timeout_ms < 0) cv_done_.wait(lk, ready);
  else if (!cv_done_.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return false;
  *out = std::move(done_[ticket]);
  done_.erase(ticket);
  return true;
}

size_t Server::peek_len(uint64_t ticket) {
  std::lock_guard<std::mutex> lk(mu_);
  auto it = done_.find(ticket);
  return it == done_.end() ? 0 : it->second.bytes.size();
}

uint64_t Server::cached_bytes() {
  std::lock_guard<std::mutex> lk(mu_);
  return bytes_;
}

int Server::prewarm(uint32_t log2, int count) {
  std::unique_lock<std::mutex> lk(mu_);
  std::vector<std::unique_ptr<Setup>> held;  // taken so that acquire builds new ones
  const uint64_t need = Setup::estimate_bytes(log2);
  try {
    while ((int)(idle_[log2].size() + held.size()) < count) {
      // build only into free room: prewarming never evicts a cached setup
      if (idle_[log2].empty() && bytes_ + need > budget_) break;
      std::unique_ptr<Setup> s = acquire(log2, lk, false);
      if (!s) break;
      held.push_back(std::move(s));
    }
  } catch (...) {
    for (auto& s : held) release(std::move(s));
    throw;
  }
  for (auto& s : held) release(std::move(s));
  return (int)idle_[log2].size();
}

// Called with the lock held; may drop it while constructing a setup.
std::unique_ptr<Setup> Server::acquire(uint32_t log2, std::unique_lock<std::mutex>& lk, bool wait) {
  for (;;) {
    if (stop_) return nullptr;
    auto it = idle_.find(log2);
    if (it != idle_.end() && !it->second.empty()) {
      std::unique_ptr<Setup> s = std::move(it->second.back().setup);
      it->second.pop_back();
      busy_++;
      return s;
    }
    const uint64_t need = Setup::estimate_bytes(log2);
    // evict idle setups until it fits: the largest first (least recently used
    // among equals).  Small setups free little room and are the cheapest to
    // keep, and rebuilding one would stall a small job far longer than its
    // proof takes.
    while (bytes_ + need > budget_) {
      uint32_t victim = 0;
      size_t vi = 0;
      uint64_t oldest = UINT64_MAX, biggest = 0;
      for (auto& kv : idle_)
        for (size_t i = 0; i < kv.second.size(); i++) {
          const uint64_t sz = kv.second[i].setup->device_bytes;
          if (sz > biggest || (sz == biggest && kv.second[i].last_use < oldest)) {
            biggest = sz;
            oldest = kv.second[i].last_use;
            victim = kv.first;
            vi = i;
          }
        }
      if (oldest == UINT64_MAX) break;  // nothing idle to evict
      auto& vec = idle_[victim];
      bytes_ -= vec[vi].setup->device_bytes;
      vec.erase(vec.begin() + (long)vi);  // frees the device buffers
    }
    if (bytes_ + need <= budget_) {
      bytes_ += need;  // reserved while constructing, corrected afterwards
      lk.unlock();
      std::unique_ptr<Setup> s;
      std::string err;
      try {
        int least = 0, greatest = 0;
        CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        s.reset(new Setup(device_, log2, log2 <= kSmallLog2 ? greatest : least));
      } catch (const std::exception& e) {
        err = e.what();
      }
      lk.lock();
      bytes_ -= need;
      if (!s) throw std::runtime_error("setup for 2^" + std::to_string(log2) + " failed: " + err);
      bytes_ += s->device_bytes;
      busy_++;
      return s;
    }
    if (busy_ == 0)  // nothing in flight will ever free memory for this job
      throw std::runtime_error("a 2^" + std::to_string(log2) + " proof does not fit the HBM budget");
    if (!wait) return nullptr;
    // every byte is held by proofs in flight: wait for one to finish
    cv_mem_.wait(lk);
  }
}

void Server::release(std::unique_ptr<Setup> s) {
  const uint32_t log2 = s->log2;
  busy_--;
  idle_[log2].push_back(Cached{std::move(s), ++use_clock_});
  cv_mem_.notify_all();
}

void Server::worker(bool small_only) {
  cudaSetDevice(device_);
  std::unique_lock<std::mutex> lk(mu_);
  for (;;) {
    size_t idx = 0;
    cv_jobs_.wait(lk, [&] { return stop_ || (idx = pick(small_only)) < queue_.size(); });
    if (stop_) return;
    Job job = std::move(queue_[idx]);
    queue_.erase(queue_.begin() + (long)idx);
    JobResult r;
    std::unique_ptr<Setup> s;
    try {
      s = acquire(job.log2, lk);
    } catch (const std::exception& e) {
      r.status = FLOCK_ERR_CAPACITY;
      r.error = e.what();
    }
    if (stop_ && !s) return;
    if (s) s->grid_sms = n_slots_ >= 3 && job.log2 > kSmallLog2 ? s->sms - kReservedSms : 0;
    const auto t_run = Clock::now();
    if (s) {
      lk.unlock();
      try {
        if (job.has_blocks) {
          const size_t n = (size_t)1 << job.log2;
          if (!s->blocks_buf)
            CK(cudaMallocAsync(reinterpret_cast<void**>(&s->blocks_buf), n * 25 * sizeof(uint32_t), s->st));
          CK(cudaMemcpyAsync(s->blocks_buf, job.blocks.data(), n * 25 * sizeof(uint32_t), cudaMemcpyHostToDevice,
                             s->st));
          r.bytes = s->prove(nullptr, s->blocks_buf, n, job.domain);
        } else {
          r.bytes = s->prove(&job.seed, nullptr, 0, job.domain);
        }
        r.status = FLOCK_OK;
        self_check(*s, job.domain, r);
      } catch (const CudaError& e) {
        r.status = FLOCK_ERR_CUDA;
        r.error = e.what();
      } catch (const std::exception& e) {
        r.status = FLOCK_ERR_INTERNAL;
        r.error = e.what();
      }
      lk.lock();
      release(std::move(s));
    }
    const auto t_end = Clock::now();
    auto ms = [](Clock::duration d) { return std::chrono::duration<double, std::milli>(d).count(); };
    r.queue_ms = ms(t_run - job.submitted);
    r.run_ms = ms(t_end - t_run);
    r.latency_ms = ms(t_end - job.submitted);
    done_[job.ticket] = std::move(r);
    cv_done_.notify_all();
  }
}

}  // namespace flock
