// Host memcpy of a few large arrays on the host's cores (staging to and from
// pinned memory): every copy is cut into pieces of 8 MB shared by the threads.
#pragma once
#include <sys/mman.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <initializer_list>
#include <thread>
#include <vector>

// Pinned result blocks shared with the batch engine (csrc/refine.cu): a block
// of at least `bytes` held by `refs` results (nullptr below the pool's minimum
// size or when the pool is full), and the release of one holder's share by
// any address inside the block.  (Global names: the batch engine's unit
// renames the gqm namespace.)
char *gqm_pinned_take(size_t bytes, int refs);
bool gqm_pinned_give(const void *p);

struct HostCopy {
  void *dst;
  const void *src;
  size_t bytes;
};

static inline void host_copy(std::initializer_list<HostCopy> list) {
  constexpr size_t kPiece = 8u << 20;
  std::vector<HostCopy> pieces;
  for (const HostCopy &c : list)
    for (size_t o = 0; o < c.bytes; o += kPiece)
      pieces.push_back({(char *)c.dst + o, (const char *)c.src + o, std::min(kPiece, c.bytes - o)});
  int nt = (int)std::min<size_t>(pieces.size(), std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
  if (nt <= 1) {
    for (const HostCopy &c : pieces) memcpy(c.dst, c.src, c.bytes);
    return;
  }
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&, t] {
      for (size_t k = t; k < pieces.size(); k += nt) memcpy(pieces[k].dst, pieces[k].src, pieces[k].bytes);
    });
  for (auto &th : pool) th.join();
}

// host_copy into one contiguous destination, with the destination handed on
// while the copy runs: `ready(offset, bytes)` is called (on the calling
// thread) for every range [offset, offset + bytes) of the destination whose
// copy is complete, in order, at least `step` bytes at a time, so that the
// caller can start its upload of the front while the back is still being
// copied.  The list's destinations must follow one another from dst_base on,
// in ascending order (gaps between them are handed on with their neighbours);
// the pieces are taken in order by the worker threads and the calling thread.
template <class List, class Ready>
static inline void host_copy_streamed(const List &list, char *dst_base, size_t step, Ready ready) {
  constexpr size_t kPiece = 4u << 20;
  std::vector<HostCopy> pieces;
  for (const HostCopy &c : list)
    for (size_t o = 0; o < c.bytes; o += kPiece)
      pieces.push_back({(char *)c.dst + o, (const char *)c.src + o, std::min(kPiece, c.bytes - o)});
  const size_t np = pieces.size();
  std::vector<std::atomic<int>> done(np);
  for (auto &d : done) d.store(0);
  std::atomic<size_t> next{0};
  auto work = [&] {
    for (size_t k = next.fetch_add(1); k < np; k = next.fetch_add(1)) {
      memcpy(pieces[k].dst, pieces[k].src, pieces[k].bytes);
      done[k].store(1, std::memory_order_release);
    }
  };
  const int nt = (int)std::min<size_t>(np, std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(work);
  // the calling thread hands on the completed front, and copies when it has nothing to hand on
  size_t front = 0;         // pieces known complete
  size_t handed = 0;        // destination bytes handed on
  size_t complete_end = 0;  // destination end of the completed prefix
  while (front < np || handed < complete_end) {
    size_t k = front;
    while (k < np && done[k].load(std::memory_order_acquire)) {
      complete_end = (size_t)((char *)pieces[k].dst + pieces[k].bytes - dst_base);
      ++k;
    }
    front = k;
    if (complete_end - handed >= step || (front == np && complete_end > handed)) {
      ready(handed, complete_end - handed);
      handed = complete_end;
      continue;
    }
    const size_t j = next.fetch_add(1);
    if (j < np) {
      memcpy(pieces[j].dst, pieces[j].src, pieces[j].bytes);
      done[j].store(1, std::memory_order_release);
    } else {
      std::this_thread::yield();
    }
  }
  for (auto &th : pool) th.join();
}

// Transparent huge pages for a large host array that has not been touched yet
// (a result array just allocated): the first-touch page faults of the copies
// into it then come in 2 MB steps instead of 4 KB ones, which roughly halves
// the time of unpacking a result of a few hundred MB.  Only the page-aligned
// interior is advised; the call is a hint and its failure is harmless.
static inline void advise_huge(void *p, size_t bytes) {
  constexpr size_t kMin = 4u << 20;
  if (!p || bytes < kMin) return;
  const uintptr_t a = ((uintptr_t)p + 4095) & ~(uintptr_t)4095;
  const uintptr_t e = ((uintptr_t)p + bytes) & ~(uintptr_t)4095;
  if (e > a) madvise((void *)a, e - a, MADV_HUGEPAGE);
}
