// Stand-in for schaapcommon's StaticFor as DP3's DDECal sources use it: the
// range [begin, end) is cut into n contiguous chunks, chunk t = [begin +
// (end - begin) t / n, begin + (end - begin) (t + 1) / n), n = min(thread
// limit, range size), each run on its own thread of the pool (f(begin, end)
// or f(begin, end, thread)). With one chunk the loop runs inline on the
// calling thread, so a caller that limits itself to one thread gets a fixed
// summation order. Only for building DP3's sources outside a DP3 tree.
#ifndef DP3B200_STANDIN_SCHAAPCOMMON_THREADING_STATICFOR_H
#define DP3B200_STANDIN_SCHAAPCOMMON_THREADING_STATICFOR_H

#include <algorithm>
#include <cstddef>
#include <type_traits>

#include "threadpool.h"

namespace schaapcommon {

template <typename Iter>
class StaticFor {
 public:
  template <typename F>
  void Run(Iter begin, Iter end, F&& f) {
    ConstrainedRun(begin, end, ThreadPool::GetInstance().NThreads(), std::forward<F>(f));
  }

  template <typename F>
  void ConstrainedRun(Iter begin, Iter end, size_t max_threads, F&& f) {
    if (end <= begin) return;
    const size_t range = size_t(end - begin);
    const size_t n = std::max<size_t>(1, std::min<size_t>(max_threads, range));
    auto chunk = [&](size_t t) {
      const Iter b = begin + Iter(range * t / n);
      const Iter e = begin + Iter(range * (t + 1) / n);
      if constexpr (std::is_invocable_v<F, Iter, Iter, size_t>)
        f(b, e, t);
      else
        f(b, e);
    };
    if (n == 1) {
      chunk(0);
      return;
    }
    ThreadPool::GetInstance().Run(n, chunk);
  }
};

template <typename Iter, typename F>
void RunStaticFor(Iter begin, Iter end, F&& f) {
  StaticFor<Iter>().Run(begin, end, std::forward<F>(f));
}

template <typename Iter, typename F>
void RunConstrainedStaticFor(Iter begin, Iter end, size_t max_threads, F&& f) {
  StaticFor<Iter>().ConstrainedRun(begin, end, max_threads, std::forward<F>(f));
}

}  // namespace schaapcommon

#endif
