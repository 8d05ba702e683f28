// Host memcpy of a few large arrays on the host's cores (staging to and from
// pinned memory): every copy is cut into pieces of 8 MB shared by the threads.
#pragma once
#include <algorithm>
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
