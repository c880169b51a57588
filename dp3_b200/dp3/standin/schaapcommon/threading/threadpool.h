// Stand-in for schaapcommon's thread pool as DP3's DDECal sources use it: a
// process-wide pool (GetInstance) of NThreads() workers that runs n tasks in
// parallel and waits for them. A task that itself asks for parallel work
// (a StaticFor inside a StaticFor, as DP3's RecursiveFor allows) gets fresh
// threads for it instead of the pool's. Only for building DP3's sources
// outside a DP3 tree; a DP3 build uses the real schaapcommon.
#ifndef DP3B200_STANDIN_SCHAAPCOMMON_THREADING_THREADPOOL_H
#define DP3B200_STANDIN_SCHAAPCOMMON_THREADING_THREADPOOL_H

#include <condition_variable>
#include <cstddef>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace schaapcommon {

class ThreadPool {
 public:
  static ThreadPool& GetInstance() {
    static ThreadPool pool;
    return pool;
  }
  ~ThreadPool() { Stop(); }

  size_t NThreads() const { return n_threads_; }

  // Replaces the workers by n of them (n >= 1). Not while tasks run.
  void SetNThreads(size_t n) {
    if (n < 1) n = 1;
    Stop();
    n_threads_ = n;
    stop_ = false;
    // A new worker waits for the next job, not for the ones before it.
    const size_t generation = generation_;
    for (size_t i = 1; i < n; ++i)
      workers_.emplace_back([this, i, generation] { WorkerLoop(i, generation); });
  }

  // Runs f(task) for task = 0 .. n_tasks - 1 (n_tasks <= NThreads()), task 0
  // on the calling thread, and waits for all of them.
  void Run(size_t n_tasks, const std::function<void(size_t)>& f) {
    if (n_tasks <= 1) {
      if (n_tasks == 1) f(0);
      return;
    }
    if (InWorker() || n_tasks > n_threads_) {  // nested or oversized: own threads
      std::vector<std::thread> extra;
      for (size_t t = 1; t < n_tasks; ++t) extra.emplace_back([&f, t] { f(t); });
      f(0);
      for (std::thread& th : extra) th.join();
      return;
    }
    std::unique_lock<std::mutex> lock(mu_);
    job_ = &f;
    job_tasks_ = n_tasks;
    pending_ = n_tasks - 1;
    ++generation_;
    cv_.notify_all();
    lock.unlock();
    InWorker() = true;
    f(0);
    InWorker() = false;
    lock.lock();
    done_cv_.wait(lock, [this] { return pending_ == 0; });
    job_ = nullptr;
  }

 private:
  ThreadPool() { SetNThreads(std::thread::hardware_concurrency()); }

  static bool& InWorker() {
    thread_local bool in_worker = false;
    return in_worker;
  }

  void WorkerLoop(size_t index, size_t seen) {
    InWorker() = true;
    std::unique_lock<std::mutex> lock(mu_);
    while (true) {
      cv_.wait(lock, [&] { return stop_ || generation_ != seen; });
      if (stop_) return;
      seen = generation_;
      if (index >= job_tasks_) continue;
      const std::function<void(size_t)>* job = job_;
      lock.unlock();
      (*job)(index);
      lock.lock();
      if (--pending_ == 0) done_cv_.notify_all();
    }
  }

  void Stop() {
    {
      std::lock_guard<std::mutex> lock(mu_);
      stop_ = true;
      cv_.notify_all();
    }
    for (std::thread& t : workers_) t.join();
    workers_.clear();
  }

  size_t n_threads_ = 1;
  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(size_t)>* job_ = nullptr;
  size_t job_tasks_ = 0;
  size_t pending_ = 0;
  size_t generation_ = 0;
  bool stop_ = false;
};

}  // namespace schaapcommon

#endif
