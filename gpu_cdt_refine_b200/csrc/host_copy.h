// Host memcpy of a few large arrays on the host's cores (staging to and from
// pinned memory): every copy is cut into pieces of 8 MB shared by the threads.
#pragma once
#include <sys/mman.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <initializer_list>
#include <thread>
#include <vector>

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
