// Host-side parallel loops and sort on std::thread, with results that do not
// depend on the number of threads (fixed chunking, deterministic splitters).
// Used by graph loading and the workload generators, whose inputs reach 2^28
// edges.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstddef>
#include <cstdint>
#include <thread>
#include <vector>

namespace dsm {

inline unsigned host_threads() {
  const unsigned hw = std::thread::hardware_concurrency();
  return std::max(1u, std::min(hw ? hw : 1u, 64u));
}

// fn(chunk) for chunk in [0, nchunks), chunks taken dynamically by the threads.
template <class Fn>
void parallel_chunks(size_t nchunks, Fn fn, unsigned nt = 0) {
  if (nt == 0) nt = host_threads();
  nt = (unsigned)std::min<size_t>(nt, nchunks);
  if (nt <= 1) {
    for (size_t c = 0; c < nchunks; ++c) fn(c);
    return;
  }
  std::atomic<size_t> next{0};
  auto work = [&]() {
    for (size_t c; (c = next.fetch_add(1)) < nchunks;) fn(c);
  };
  std::vector<std::thread> th;
  for (unsigned t = 1; t < nt; ++t) th.emplace_back(work);
  work();
  for (auto &t : th) t.join();
}

// fn(lo, hi) over [0, n) in fixed chunks of `grain`.
template <class Fn>
void parallel_for(size_t n, size_t grain, Fn fn) {
  if (n == 0) return;
  grain = std::max<size_t>(grain, 1);
  parallel_chunks((n + grain - 1) / grain, [&](size_t c) { fn(c * grain, std::min(n, (c + 1) * grain)); });
}

// Sample sort: splitters from a fixed-stride sample, elements scattered into
// buckets (two counting passes), buckets sorted in parallel.  The result is
// the sorted sequence, identical to std::sort's.
template <class T>
void parallel_sort(std::vector<T> &v) {
  const size_t n = v.size();
  const unsigned nt = host_threads();
  if (n < (1u << 20) || nt == 1) {
    std::sort(v.begin(), v.end());
    return;
  }
  const size_t nb = 1024;
  const size_t ns = 64 * nb;
  std::vector<T> sample(ns);
  for (size_t i = 0; i < ns; ++i) sample[i] = v[(i * (n / ns)) + (n / ns) / 2];
  std::sort(sample.begin(), sample.end());
  std::vector<T> split(nb - 1);
  for (size_t k = 1; k < nb; ++k) split[k - 1] = sample[k * 64];
  auto bucket = [&](const T &x) { return (size_t)(std::upper_bound(split.begin(), split.end(), x) - split.begin()); };
  const size_t grain = 1u << 20;
  const size_t nchunks = (n + grain - 1) / grain;
  std::vector<uint64_t> cnt(nchunks * nb, 0);
  parallel_chunks(nchunks, [&](size_t c) {
    uint64_t *h = cnt.data() + c * nb;
    for (size_t i = c * grain, e = std::min(n, (c + 1) * grain); i < e; ++i) h[bucket(v[i])]++;
  });
  // bucket-major prefix: bucket b's region holds chunk 0's, then chunk 1's ...
  std::vector<uint64_t> bstart(nb + 1, 0);
  {
    uint64_t acc = 0;
    for (size_t b = 0; b < nb; ++b) {
      bstart[b] = acc;
      for (size_t c = 0; c < nchunks; ++c) {
        uint64_t x = cnt[c * nb + b];
        cnt[c * nb + b] = acc;
        acc += x;
      }
    }
    bstart[nb] = acc;
  }
  std::vector<T> out(n);
  parallel_chunks(nchunks, [&](size_t c) {
    uint64_t *h = cnt.data() + c * nb;
    for (size_t i = c * grain, e = std::min(n, (c + 1) * grain); i < e; ++i) out[h[bucket(v[i])]++] = v[i];
  });
  parallel_chunks(nb, [&](size_t b) { std::sort(out.begin() + bstart[b], out.begin() + bstart[b + 1]); });
  v.swap(out);
}

}  // namespace dsm
