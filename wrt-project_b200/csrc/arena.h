// arena.h -- first-fit sub-allocator over one fixed range of device memory.
//
// The serving loop reserves its whole HBM budget with one cudaMalloc at
// start-up and carves request state (volumes, layer pairs, outputs, spline
// lines) out of it here: cudaMalloc / cudaFree would synchronise the device
// between batches and defeat the overlap of consecutive launches.  Offsets
// are aligned to 256 bytes; freed blocks are coalesced with their neighbours.
// Not thread-safe: the server calls it under its own lock.  Pure C++ (no CUDA)
// so it is tested on the CPU.
#pragma once
#include <stddef.h>

#include <iterator>
#include <map>
#include <unordered_map>

namespace wrt {

class Arena {
 public:
  static constexpr size_t kAlign = 256;

  void reset(size_t capacity) {
    cap_ = capacity & ~(kAlign - 1);
    free_.clear();
    live_.clear();
    used_ = peak_ = 0;
    if (cap_) free_[0] = cap_;
  }
  static size_t round_up(size_t bytes) { return (bytes + kAlign - 1) & ~(kAlign - 1); }

  // First fit.  Returns false (and leaves the arena unchanged) when no free
  // block is large enough.
  bool alloc(size_t bytes, size_t *offset) {
    const size_t need = round_up(bytes ? bytes : 1);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < need) continue;
      const size_t off = it->first, rest = it->second - need;
      free_.erase(it);
      if (rest) free_[off + need] = rest;
      live_[off] = need;
      used_ += need;
      if (used_ > peak_) peak_ = used_;
      *offset = off;
      return true;
    }
    return false;
  }

  // Returns false for an offset that is not a live block.
  bool release(size_t offset) {
    auto lv = live_.find(offset);
    if (lv == live_.end()) return false;
    size_t off = offset, size = lv->second;
    live_.erase(lv);
    used_ -= size;
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + size == next->first) {
      size += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += size;
        return true;
      }
    }
    free_[off] = size;
    return true;
  }

  // Would a request of these block sizes fit right now (first fit, in order)?
  template <typename It>
  bool fits(It first, It last) const {
    std::map<size_t, size_t> f = free_;
    for (; first != last; ++first) {
      const size_t need = round_up(*first ? *first : 1);
      bool ok = false;
      for (auto it = f.begin(); it != f.end(); ++it) {
        if (it->second < need) continue;
        const size_t off = it->first, rest = it->second - need;
        f.erase(it);
        if (rest) f[off + need] = rest;
        ok = true;
        break;
      }
      if (!ok) return false;
    }
    return true;
  }

  size_t capacity() const { return cap_; }
  size_t used() const { return used_; }
  size_t peak() const { return peak_; }
  size_t live_blocks() const { return live_.size(); }
  size_t free_blocks() const { return free_.size(); }
  size_t largest_free() const {
    size_t m = 0;
    for (auto &kv : free_) m = kv.second > m ? kv.second : m;
    return m;
  }

 private:
  size_t cap_ = 0, used_ = 0, peak_ = 0;
  std::map<size_t, size_t> free_;           // offset -> bytes
  std::unordered_map<size_t, size_t> live_;  // offset -> bytes
};

}  // namespace wrt
