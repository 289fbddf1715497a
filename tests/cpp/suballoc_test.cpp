// CPU test of the library's range allocator (dcsr_b200/csrc/suballoc.hpp):
// fixed cases for best fit, splitting, merging and region boundaries, then a
// seeded random run of allocations, frees and event completions that checks
// after every step that no two handed-out blocks overlap, every block lies
// aligned inside one region, event reference counts stay consistent, and
// that once every event has completed and every block is returned the free
// space merges back to one block per region.  Prints "ok" on success.
#include <cstdio>
#include <cstdlib>
#include <map>
#include <random>
#include <vector>

#include "suballoc.hpp"

using dcsr::RangeAlloc;

#define CHECK(c)                                                      \
  do {                                                                \
    if (!(c)) {                                                       \
      std::fprintf(stderr, "check failed at line %d: %s\n", __LINE__, #c); \
      std::exit(1);                                                   \
    }                                                                 \
  } while (0)

struct Events {
  std::vector<int> refs;
  std::vector<bool> done;
  int make() {
    refs.push_back(1);
    done.push_back(false);
    return (int)refs.size() - 1;
  }
  void drop(int e) {
    CHECK(e >= 0 && e < (int)refs.size() && refs[e] > 0);
    refs[e]--;
  }
  void retain(int e) {
    CHECK(e >= 0 && e < (int)refs.size() && refs[e] > 0);
    refs[e]++;
  }
};

static void fixed_cases() {
  Events ev;
  RangeAlloc ra;
  ra.add_region(0x10000, 1 << 20);
  CHECK(ra.total() == (1u << 20) && ra.free_blocks() == 1);
  auto a = ra.alloc(1000, [&](int e) { ev.retain(e); });
  CHECK(a.addr == 0x10000 && a.ev == -1);  // rounded to 1024
  auto b = ra.alloc(256, [&](int e) { ev.retain(e); });
  CHECK(b.addr == 0x10000 + 1024);
  auto c = ra.alloc(4096, [&](int e) { ev.retain(e); });
  CHECK(c.addr == 0x10000 + 1024 + 256);
  CHECK(ra.in_use() == 1024 + 256 + 4096);
  // free a settled: it does not merge with b (in use); b settled merges a and b
  CHECK(ra.free(a.addr, -1));
  CHECK(!ra.free(a.addr, -1));  // twice: not ours any more
  CHECK(ra.free(b.addr, -1));
  CHECK(ra.free_blocks() == 2);  // [a+b] and the tail after c
  // best fit: a 1280-byte request takes the merged 1280-byte hole exactly
  auto d = ra.alloc(1280, [&](int e) { ev.retain(e); });
  CHECK(d.addr == 0x10000 && ra.free_blocks() == 1);
  // pending block: freed with an event, taken only when nothing settled fits
  const int e1 = ev.make();
  CHECK(ra.free(c.addr, e1));
  auto f = ra.alloc(64, [&](int e) { ev.retain(e); });  // settled tail fits: no wait
  CHECK(f.ev == -1 && f.addr != c.addr);
  auto g = ra.alloc((1 << 20) - 1280 - 4096 - 256 + 1, [&](int e) { ev.retain(e); });  // larger than the tail
  CHECK(g.addr == 0);
  auto h = ra.alloc(1024, [&](int e) { ev.retain(e); });  // the settled tail, before c's pending block
  CHECK(h.addr != 0 && h.ev == -1 && h.addr != c.addr);
  // settle: c's event completes, its block merges with its settled neighbours
  ev.done[e1] = true;
  ra.settle([&](int e) { return (bool)ev.done[e]; }, [&](int e) { ev.drop(e); });
  if (h.ev >= 0) ev.drop(h.ev);
  CHECK(ra.free(d.addr, -1) && ra.free(f.addr, -1) && ra.free(h.addr, -1));
  CHECK(ra.free_blocks() == 1 && ra.free_bytes() == ra.total());
  CHECK(ev.refs[e1] == 0);

  // a pending block split on allocation: the remainder keeps the event
  RangeAlloc rb;
  Events ev2;
  rb.add_region(0x100000, 8192);
  auto x = rb.alloc(8192, [&](int e) { ev2.retain(e); });
  CHECK(x.addr == 0x100000);
  const int e2 = ev2.make();
  CHECK(rb.free(x.addr, e2));
  auto y = rb.alloc(2048, [&](int e) { ev2.retain(e); });
  CHECK(y.addr == 0x100000 && y.ev == e2 && ev2.refs[e2] == 2);  // caller's and the remainder's
  ev2.drop(y.ev);                                                  // the caller waited
  ev2.done[e2] = true;
  rb.settle([&](int e) { return (bool)ev2.done[e]; }, [&](int e) { ev2.drop(e); });
  CHECK(ev2.refs[e2] == 0);
  CHECK(rb.free(y.addr, -1) && rb.free_blocks() == 1);

  // two regions whose addresses touch are never merged
  RangeAlloc rc;
  rc.add_region(0x200000, 4096);
  rc.add_region(0x201000, 4096);
  CHECK(rc.free_blocks() == 2);
  CHECK(rc.alloc(8192, [](int) {}).addr == 0);
  // unaligned region edges are trimmed to the alignment
  RangeAlloc rd;
  rd.add_region(0x300010, 1000);
  CHECK(rd.total() == 512 && rd.alloc(512, [](int) {}).addr == 0x300100);
}

static void random_run(unsigned seed) {
  std::mt19937_64 rng(seed);
  Events ev;
  RangeAlloc ra;
  struct R {
    uint64_t base, size;
  };
  std::vector<R> regions = {{0x1000000, 3u << 20}, {0x9000000, 5u << 20}, {0x20000000, 1u << 20}};
  for (auto &r : regions) ra.add_region(r.base, r.size);
  std::map<uint64_t, uint64_t> live;  // addr -> requested bytes
  std::vector<int> open_events;
  for (int step = 0; step < 20000; step++) {
    const int op = (int)(rng() % 10);
    if (op < 5) {
      const uint64_t want = 1 + rng() % (rng() % 4 == 0 ? (512u << 10) : 8192u);
      const bool allow_pending = rng() % 3 != 0;
      auto g = ra.alloc(want, [&](int e) { ev.retain(e); }, allow_pending);
      if (!allow_pending) CHECK(g.ev == -1);
      if (g.addr) {
        CHECK(g.addr % RangeAlloc::ALIGN == 0);
        int in = 0;
        for (auto &r : regions) in += g.addr >= r.base && g.addr + want <= r.base + r.size;
        CHECK(in == 1);
        auto nx = live.lower_bound(g.addr);
        if (nx != live.end()) CHECK(g.addr + want <= nx->first);
        if (nx != live.begin()) {
          auto pv = std::prev(nx);
          CHECK(pv->first + pv->second <= g.addr);
        }
        if (g.ev >= 0) ev.drop(g.ev);  // the caller's wait done
        live[g.addr] = want;
      }
    } else if (op < 8 && !live.empty()) {
      auto it = live.begin();
      std::advance(it, rng() % live.size());
      int e = -1;
      if (rng() % 2) {
        e = ev.make();
        open_events.push_back(e);
      }
      CHECK(ra.free(it->first, e));
      live.erase(it);
    } else if (!open_events.empty()) {
      const size_t k = rng() % open_events.size();
      ev.done[open_events[k]] = true;
      open_events.erase(open_events.begin() + k);
      ra.settle([&](int e) { return (bool)ev.done[e]; }, [&](int e) { ev.drop(e); });
    }
    uint64_t used = 0;
    for (auto &kv : live) used += (kv.second + 255) / 256 * 256;
    CHECK(ra.in_use() == used);
  }
  for (auto &kv : live) CHECK(ra.free(kv.first, -1));
  for (int e : open_events) ev.done[e] = true;
  ra.settle([&](int e) { return (bool)ev.done[e]; }, [&](int e) { ev.drop(e); });
  CHECK(ra.free_blocks() == regions.size());
  CHECK(ra.free_bytes() == ra.total() && ra.pending_blocks() == 0);
  for (int r : ev.refs) CHECK(r == 0);
}

int main() {
  fixed_cases();
  for (unsigned seed = 1; seed <= 8; seed++) random_run(seed);
  std::printf("ok\n");
  return 0;
}
