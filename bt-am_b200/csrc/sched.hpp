// Admission queue of the job server (pure host C++, no CUDA).
//
// Jobs wait in arrival order.  A worker slot that frees up takes the first
// waiting job whose device-memory footprint fits the budget next to the jobs
// already running, with one rule against starvation: a job behind the head of
// the queue may start before the head only if it leaves room for the head,
// i.e. running + head + job <= budget.  So the head is admitted as soon as the
// jobs running at the moment it reached the head have drained, whatever keeps
// arriving behind it, while small jobs fill the memory and slots the head
// cannot use yet (backfilling with a reservation for the head).
#pragma once

#include <cstddef>
#include <cstdint>
#include <deque>
#include <vector>

namespace btam {

struct QueuedJob {
  long long id;
  std::size_t bytes;  // estimated device footprint
};

class AdmissionQueue {
 public:
  explicit AdmissionQueue(std::size_t budget) : budget_(budget) {}

  std::size_t budget() const { return budget_; }
  std::size_t in_use() const { return in_use_; }
  std::size_t waiting() const { return q_.size(); }

  // A job larger than the whole budget can never run; the caller rejects it.
  bool fits_ever(std::size_t bytes) const { return bytes <= budget_; }

  void push(long long id, std::size_t bytes) { q_.push_back(QueuedJob{id, bytes}); }

  // The next job to start under the rule above, removed from the queue and
  // counted in the memory in use; -1 if none may start now.
  long long admit() {
    if (q_.empty()) return -1;
    const std::size_t head = q_.front().bytes;
    if (in_use_ + head <= budget_) return take(0);
    for (std::size_t k = 1; k < q_.size(); ++k)
      if (in_use_ + head + q_[k].bytes <= budget_) return take(k);
    return -1;
  }

  // A running job finished: its memory returns to the budget.
  void release(std::size_t bytes) { in_use_ = bytes > in_use_ ? 0 : in_use_ - bytes; }

 private:
  long long take(std::size_t k) {
    QueuedJob j = q_[k];
    q_.erase(q_.begin() + (std::ptrdiff_t)k);
    in_use_ += j.bytes;
    return j.id;
  }
  std::size_t budget_;
  std::size_t in_use_ = 0;
  std::deque<QueuedJob> q_;
};

}  // namespace btam
