// A small pool of host threads for the per-member work of a batch (the forward, coordinate,
// tangent and set-up calls of independent contexts, each issuing its own launches on its own
// stream): the host's launch overhead is what those calls cost, so spreading them over threads
// shortens the rounds of a batched run.
#pragma once

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace dmk {

class HostPool {
 public:
  // n_threads workers besides the calling thread; every worker selects `device` first
  HostPool(int n_threads, int device);
  ~HostPool();
  HostPool(const HostPool&) = delete;
  HostPool& operator=(const HostPool&) = delete;

  // f(k) for k = 0 .. n-1 on the workers and the calling thread; returns when all have run.
  // f returns 0 or an error code; the result is 0, or the code of the lowest failing k with the
  // library's error message of that call in *msg.
  int run(int n, const std::function<int(int)>& f, std::string* msg);

 private:
  void work(int device);
  void drain();

  std::vector<std::thread> threads_;
  std::mutex m_;
  std::condition_variable start_, done_;
  const std::function<int(int)>* job_ = nullptr;
  int n_ = 0;
  std::atomic<int> next_{0};
  int busy_ = 0;
  uint64_t generation_ = 0;
  bool stop_ = false;
  std::vector<int> rc_;
  std::vector<std::string> msg_;
};

}  // namespace dmk
