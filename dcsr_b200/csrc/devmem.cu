// Device memory of the library: every pool, schedule, scratch arena and
// staging buffer is allocated by dev_alloc and returned by dev_free.
//
// dcsr_pool_reserve maps regions up front (per device); dev_alloc carves
// blocks from them through RangeAlloc (suballoc.hpp) and only falls back to
// the driver's stream-ordered allocator when no region block fits (counted).
// Stream order: dev_free records an event on the freeing stream and the
// block stays pending until that event completes; an allocation that takes
// a pending block makes its own stream wait on the event.  Inside a stream
// capture nothing is taken from the regions (a captured allocation is the
// graph's), and a region block freed inside a capture is an error.
#include <atomic>
#include <cstdio>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "internal.cuh"
#include "suballoc.hpp"

namespace dcsr {
namespace {

constexpr int MAX_DEVICES = 64;

struct DeviceRegions {
  RangeAlloc ra;
  std::vector<cudaEvent_t> evs;  // event table; blocks hold ids with reference counts
  std::vector<int> refs;
  std::vector<int> spare_ids;
  long long fallback = 0;  // allocations the regions could not hold
};

std::mutex g_mem_mu;
DeviceRegions g_regions[MAX_DEVICES];
std::atomic<int> g_region_devices{0};  // devices with at least one region (skip the search when none)

int take_event(DeviceRegions &D) {
  int id;
  if (!D.spare_ids.empty()) {
    id = D.spare_ids.back();
    D.spare_ids.pop_back();
  } else {
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return -1;
    id = (int)D.evs.size();
    D.evs.push_back(e);
    D.refs.push_back(0);
  }
  D.refs[id] = 1;
  return id;
}

void drop_event(DeviceRegions &D, int id) {
  if (--D.refs[id] == 0) D.spare_ids.push_back(id);
}

bool event_done(DeviceRegions &D, int id) {
  const cudaError_t e = cudaEventQuery(D.evs[id]);
  // "not ready" is no error: leave no trace of it for the next launch check
  // (an earlier, real error stays where it is)
  if (e == cudaErrorNotReady && cudaPeekAtLastError() == cudaErrorNotReady) (void)cudaGetLastError();
  return e == cudaSuccess;
}

bool capturing(cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone;
}

}  // namespace

cudaError_t dev_alloc_raw(void **p, size_t bytes, cudaStream_t s) {
  int dev = 0;
  if (g_region_devices > 0 && cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < MAX_DEVICES &&
      !capturing(s)) {
    std::lock_guard<std::mutex> lk(g_mem_mu);
    DeviceRegions &D = g_regions[dev];
    if (D.ra.total() > 0) {
      auto retain = [&](int e) { D.refs[e]++; };
      // a settled block first (no event query, no wait); else settle what
      // has completed and take the best block, pending or not
      RangeAlloc::Got g = D.ra.pending_blocks() > 256 ? RangeAlloc::Got{} : D.ra.alloc(bytes, retain, false);
      if (!g.addr) {
        D.ra.settle([&](int e) { return event_done(D, e); }, [&](int e) { drop_event(D, e); });
        g = D.ra.alloc(bytes, retain, true);
      }
      if (g.addr) {
        if (g.ev >= 0) {
          const cudaError_t e = cudaStreamWaitEvent(s, D.evs[g.ev], 0);
          if (e != cudaSuccess) {
            D.ra.free(g.addr, g.ev);  // back, still pending on its event (the reference goes with it)
            return e;
          }
          drop_event(D, g.ev);
        }
        *p = reinterpret_cast<void *>(g.addr);
        return cudaSuccess;
      }
      D.fallback++;
    }
  }
  return cudaMallocAsync(p, bytes, s);
}

cudaError_t dev_free(void *p, cudaStream_t s) {
  if (!p) return cudaSuccess;
  if (g_region_devices > 0) {
    std::lock_guard<std::mutex> lk(g_mem_mu);
    for (DeviceRegions &D : g_regions) {
      if (D.ra.total() == 0 || !D.ra.owns(reinterpret_cast<uint64_t>(p))) continue;
      if (capturing(s)) {
        fprintf(stderr, "dcsr: a reserved-region block freed inside a stream capture is kept (not reused)\n");
        return cudaErrorStreamCaptureUnsupported;
      }
      const int id = take_event(D);
      if (id >= 0 && cudaEventRecord(D.evs[id], s) == cudaSuccess) {
        D.ra.free(reinterpret_cast<uint64_t>(p), id);
        return cudaSuccess;
      }
      // no event on this stream (another device's, or none left): wait for
      // the stream, then the block is settled at once
      if (id >= 0) drop_event(D, id);
      const cudaError_t e = cudaStreamSynchronize(s);
      if (e == cudaSuccess) D.ra.free(reinterpret_cast<uint64_t>(p), -1);
      return e;
    }
  }
  return cudaFreeAsync(p, s);
}

int reserve_regions(int64_t bytes, cudaStream_t s) {
  int dev = 0;
  DCSR_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= MAX_DEVICES) return DCSR_NOT_SUPPORTED;
  std::lock_guard<std::mutex> lk(g_mem_mu);
  DeviceRegions &D = g_regions[dev];
  const uint64_t have = D.ra.free_bytes();
  if (have >= (uint64_t)bytes) return DCSR_OK;
  const int64_t add = align_up(bytes - (int64_t)have, 2ll << 20);
  void *p = nullptr;
  DCSR_CUDA(cudaMallocAsync(&p, (size_t)add, s));  // kept for the life of the process
  DCSR_CUDA(cudaStreamSynchronize(s));
  if (D.ra.total() == 0) g_region_devices++;
  D.ra.add_region(reinterpret_cast<uint64_t>(p), (uint64_t)add);
  return DCSR_OK;
}

int region_usage(int64_t *reserved, int64_t *free_bytes, int64_t *fallback) {
  int dev = 0;
  DCSR_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= MAX_DEVICES) return DCSR_NOT_SUPPORTED;
  std::lock_guard<std::mutex> lk(g_mem_mu);
  const DeviceRegions &D = g_regions[dev];
  if (reserved) *reserved = (int64_t)D.ra.total();
  if (free_bytes) *free_bytes = (int64_t)D.ra.free_bytes();
  if (fallback) *fallback = D.fallback;
  return DCSR_OK;
}

}  // namespace dcsr
