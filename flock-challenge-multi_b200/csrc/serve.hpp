// Serving scheduler: continuous batching of proof jobs of different sizes on
// one GPU.  Jobs are admitted as proof slots and device memory free up: each
// slot is a host thread that drives one proof at a time on its own CUDA
// stream, so the kernels of up to `slots` proofs overlap on the device and
// fill each other's host round-trip gaps (the Fiat-Shamir transcript stays on
// the host).  The queue is size-aware, so that small jobs do not wait behind
// 2^19 / 2^20 proofs: a free slot takes the job with the shortest expected
// proof, aged by its waiting time (a job that has waited kAging times its own
// expected run time goes ahead of any fresh job); with 3 or more slots a
// quarter of the slots (at least one) take only small jobs (at most
// 2^kSmallLog2 compressions), and small jobs' setups run on the
// highest-priority CUDA stream.  Setups (device buffers + tables for one
// size) are cached per size and reused; admission keeps the bytes of all
// cached setups within the HBM budget, evicting idle setups (the largest
// first) when a new setup needs room.
#pragma once
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include "prover.hpp"

namespace flock {

struct JobResult {
  int status = 0;  // FLOCK_* status of the proof
  std::string error;
  std::vector<uint8_t> bytes;
  double queue_ms = 0, run_ms = 0, latency_ms = 0;
};

class Server {
 public:
  // budget: device bytes all cached setups may hold; slots: proofs in flight
  Server(int device, uint64_t budget, int slots);
  ~Server();
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;

  // blocks == nullptr: inputs generated on the device from `seed`; otherwise
  // 2^log2 x 25 u32, copied here (the caller may free them on return)
  uint64_t submit(uint32_t log2, uint64_t seed, const uint32_t* blocks, const std::string& domain);
  // true once the job finished (its result is moved out and forgotten)
  bool wait(uint64_t ticket, int timeout_ms, JobResult* out);
  // the job's proof length if finished, else 0 (leaves the result in place)
  size_t peek_len(uint64_t ticket);

  // Batched form: prove `jobs` together, in waves of as many jobs as fit the
  // HBM budget; the seeded jobs of a wave share one fused witness + commit
  // graph (batch_commit), then the remaining phases of every proof of the
  // wave run concurrently on `threads` host threads, one stream each.
  struct BatchItem {
    uint32_t log2 = 0;
    uint64_t seed = 0;
    const uint32_t* blocks = nullptr;  // or 2^log2 x 25 u32 on the host
    std::string domain;
  };
  std::vector<JobResult> prove_batch(const std::vector<BatchItem>& jobs, int threads);

  // Builds setups of size log2 until `count` of them are cached idle (as
  // many as fit the free budget: it evicts nothing); returns how many are.  Building a setup takes
  // tens of milliseconds, so a server that expects bursts of a size builds
  // them before the jobs arrive.
  int prewarm(uint32_t log2, int count);
  // self-check: verify every proof on its own setup before returning it; a
  // proof that fails gets FLOCK_ERR_VERIFY and the failed check's name
  void set_verify(bool on) { verify_ = on; }
  int slots() const { return n_slots_; }
  uint64_t budget() const { return budget_; }
  uint64_t cached_bytes();

 private:
  using Clock = std::chrono::steady_clock;
  struct Job {
    uint64_t ticket = 0;
    uint32_t log2 = 0;
    uint64_t seed = 0;
    bool has_blocks = false;
    std::vector<uint32_t> blocks;
    std::string domain;
    Clock::time_point submitted;
  };
  struct Cached {
    std::unique_ptr<Setup> setup;
    uint64_t last_use = 0;
  };

  static constexpr uint32_t kSmallLog2 = 16;
  // with an express slot, large proofs' grid-stride kernels leave this many
  // SMs free, so that a small proof's kernels need not wait for them
  static constexpr int kReservedSms = 16;
  static constexpr double kAging = 2.0;
  static double expected_ms(uint32_t log2);
  // index of the queued job a free slot takes next (queue_.size() if none)
  size_t pick(bool small_only) const;
  void worker(bool small_only);
  void self_check(Setup& s, const std::string& domain, JobResult& r);
  // wait: block until memory frees up (else return nullptr when it does not fit now)
  std::unique_ptr<Setup> acquire(uint32_t log2, std::unique_lock<std::mutex>& lk, bool wait = true);
  void release(std::unique_ptr<Setup> s);

  int device_;
  uint64_t budget_;
  std::mutex mu_;
  std::condition_variable cv_jobs_, cv_done_, cv_mem_;
  std::deque<Job> queue_;
  std::map<uint64_t, JobResult> done_;
  std::map<uint32_t, std::vector<Cached>> idle_;  // cached setups not in use, by size
  uint64_t bytes_ = 0;                            // device bytes of all setups (idle + busy)
  int busy_ = 0;                                  // setups held by proofs in flight
  uint64_t next_ticket_ = 1, use_clock_ = 0;
  bool stop_ = false;
  std::atomic<bool> verify_{false};
  int n_slots_ = 0;  // set before the slot threads start (they read it)
  std::vector<std::thread> workers_;
  std::mutex batch_mu_;  // one batch at a time
  cudaStream_t batch_st_ = nullptr;
};

}  // namespace flock
