// Stand-in for aocommon's FIFO queue as DP3's BdaSolverBuffer declares it
// (PushBack, Size, indexing from the front). Only for building DP3's sources
// outside a DP3 tree.
#ifndef DP3B200_STANDIN_AOCOMMON_QUEUE_H
#define DP3B200_STANDIN_AOCOMMON_QUEUE_H

#include <cstddef>
#include <deque>
#include <utility>

namespace aocommon {

template <typename T>
class Queue {
 public:
  void PushBack(T&& v) { q_.push_back(std::move(v)); }
  void PushBack(const T& v) { q_.push_back(v); }
  void PopFront() { q_.pop_front(); }
  size_t Size() const { return q_.size(); }
  bool Empty() const { return q_.empty(); }
  T& operator[](size_t i) { return q_[i]; }
  const T& operator[](size_t i) const { return q_[i]; }
  T& Front() { return q_.front(); }
  void Clear() { q_.clear(); }

 private:
  std::deque<T> q_;
};

}  // namespace aocommon

#endif
