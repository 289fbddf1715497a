// Range allocator over device memory regions, host-side bookkeeping only
// (no CUDA in this file, so it is unit-tested on the CPU).
//
// The library's matrix pools, schedules and scratch are carved from regions
// that dcsr_pool_reserve maps up front, so a pool growth, a repair or a
// compaction inside a timed loop never asks the driver for new device
// memory (a stream-ordered allocation that maps fresh memory measured tens
// to hundreds of milliseconds on busy hosts).  Blocks are handed out best
// fit at 256-byte alignment.  A freed block carries the caller's event id
// for the work still using it ("pending"); it is merged with free
// neighbours of its region only once the caller reports that event complete
// ("settled").  An allocation takes the smallest settled block that fits,
// else the smallest pending one, whose event it returns: the caller makes
// its stream wait on it, so reuse stays stream-ordered without a host sync.
// The caller settles lazily (when no settled block fits, or many blocks are
// pending), so most allocations query no event.
#pragma once

#include <cstdint>
#include <iterator>
#include <map>
#include <vector>

namespace dcsr {

class RangeAlloc {
 public:
  static constexpr uint64_t ALIGN = 256;
  struct Got {
    uint64_t addr = 0;  // 0: no block fits
    int ev = -1;        // event to wait on before use; its reference passes to the caller
  };

  void add_region(uint64_t base, uint64_t size) {
    const uint64_t b = (base + ALIGN - 1) / ALIGN * ALIGN;
    const uint64_t e = (base + size) / ALIGN * ALIGN;
    if (e <= b) return;
    regions_.push_back(Region{b, e - b});
    total_ += e - b;
    put_free(b, e - b, -1);
  }

  bool owns(uint64_t addr) const { return used_.count(addr) != 0; }
  uint64_t total() const { return total_; }
  uint64_t in_use() const { return in_use_; }
  uint64_t free_bytes() const { return total_ - in_use_; }
  size_t free_blocks() const { return free_.size(); }
  size_t pending_blocks() const { return pending_; }
  // Size of the largest settled block (what an allocation can take with no wait).
  uint64_t largest_settled() const {
    uint64_t m = 0;
    for (auto &kv : free_)
      if (kv.second.ev < 0 && kv.second.size > m) m = kv.second.size;
    return m;
  }

  // Settles every pending block whose event done(ev) reports complete,
  // dropping its reference through drop(ev) and merging it with settled
  // neighbours.
  template <typename Done, typename Drop>
  void settle(Done done, Drop drop) {
    std::vector<uint64_t> ready;
    for (auto &kv : free_)
      if (kv.second.ev >= 0 && done(kv.second.ev)) ready.push_back(kv.first);
    for (uint64_t a : ready) {
      auto it = free_.find(a);
      const uint64_t sz = it->second.size;
      drop(it->second.ev);
      erase(it);
      put_free(a, sz, -1);
    }
  }

  // Best fit: the smallest settled block holding `bytes` (rounded up to
  // ALIGN), else (when allow_pending) the smallest pending one.  A block
  // larger than the request is split; a pending remainder keeps the event,
  // with the reference that retain(ev) adds for it.
  template <typename Retain>
  Got alloc(uint64_t bytes, Retain retain, bool allow_pending = true) {
    const uint64_t need = bytes == 0 ? ALIGN : (bytes + ALIGN - 1) / ALIGN * ALIGN;
    if (need < bytes) return Got{};  // overflow of the rounding
    auto best = free_.end();
    for (int pass = 0; pass < (allow_pending ? 2 : 1) && best == free_.end(); pass++)
      for (auto it = free_.begin(); it != free_.end(); ++it) {
        const bool settled = it->second.ev < 0;
        if (settled != (pass == 0) || it->second.size < need) continue;
        if (best == free_.end() || it->second.size < best->second.size) best = it;
      }
    if (best == free_.end()) return Got{};
    const uint64_t a = best->first, sz = best->second.size;
    const int ev = best->second.ev;
    erase(best);
    if (sz > need) {
      if (ev >= 0) retain(ev);
      put_free(a + need, sz - need, ev);
    }
    used_[a] = need;
    in_use_ += need;
    return Got{a, ev};
  }

  // Returns a block that alloc handed out (false: not one of this
  // allocator's).  ev (or -1) is the caller's event for the work that still
  // uses the block; the block holds that reference until it is settled.
  bool free(uint64_t addr, int ev) {
    auto it = used_.find(addr);
    if (it == used_.end()) return false;
    const uint64_t sz = it->second;
    used_.erase(it);
    in_use_ -= sz;
    put_free(addr, sz, ev);
    return true;
  }

 private:
  struct Block {
    uint64_t size;
    int ev;
  };
  struct Region {
    uint64_t base, size;
  };
  std::map<uint64_t, Block>::iterator erase(std::map<uint64_t, Block>::iterator it) {
    pending_ -= it->second.ev >= 0;
    return free_.erase(it);
  }
  int region_of(uint64_t a) const {
    for (size_t i = 0; i < regions_.size(); i++)
      if (a >= regions_[i].base && a - regions_[i].base < regions_[i].size) return (int)i;
    return -1;
  }
  // A free block; a settled one is merged with the settled blocks either
  // side of it in the same region (regions are separate driver allocations
  // and are never joined, even when their addresses touch).
  void put_free(uint64_t a, uint64_t sz, int ev) {
    if (ev < 0) {
      const int r = region_of(a);
      auto nx = free_.lower_bound(a);
      if (nx != free_.end() && nx->second.ev < 0 && nx->first == a + sz && region_of(nx->first) == r) {
        sz += nx->second.size;
        nx = erase(nx);
      }
      if (nx != free_.begin()) {
        auto pv = std::prev(nx);
        if (pv->second.ev < 0 && pv->first + pv->second.size == a && region_of(pv->first) == r) {
          a = pv->first;
          sz += pv->second.size;
          erase(pv);
        }
      }
    }
    free_[a] = Block{sz, ev};
    pending_ += ev >= 0;
  }

  std::vector<Region> regions_;
  std::map<uint64_t, Block> free_;    // address -> free block
  std::map<uint64_t, uint64_t> used_;  // address -> size of a handed-out block
  uint64_t total_ = 0, in_use_ = 0;
  size_t pending_ = 0;
};

}  // namespace dcsr
