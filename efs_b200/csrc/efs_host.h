// Host-side planning helpers of the engine (plain C++17, no CUDA): the
// threaded stable radix sort that orders point lists by device index, the
// grouping of entries by target built on it, and the chunked host-thread
// loop.  Compiled into libefs.so and, on its own, into the CPU test of these
// helpers (tests/test_host_plan.py).
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <thread>
#include <vector>

namespace efs_host {

// Host threads for a loop over n items of configure-time work (1 below 64 K items).
inline unsigned host_threads(size_t n) {
    if (n < (1u << 16)) return 1;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    return (unsigned)std::min<size_t>({(size_t)std::min(hw, 16u), n >> 15});
}

// f(t, lo, hi) on T contiguous chunks of [0, n), chunk t on its own thread
// (chunk 0 on the caller's).  f must not throw.
template <class F>
void parallel_chunks(size_t n, unsigned T, F&& f) {
    if (T <= 1) { f(0u, (size_t)0, n); return; }
    std::vector<std::thread> th;
    th.reserve(T - 1);
    for (unsigned t = 1; t < T; ++t) th.emplace_back([&, t] { f(t, n * t / T, n * (t + 1) / T); });
    f(0u, (size_t)0, n / T);
    for (auto& x : th) x.join();
}

// Stable LSD radix sort of (key, value) pairs by key (11-bit digits; digits
// above the largest key are skipped; input already in key order is left
// as it is).  Each pass runs on T host threads over contiguous chunks:
// per-chunk digit counts, offsets in (digit, chunk) order, then each chunk
// scatters its items in order, which keeps the sort stable.
inline void radix_sort_pairs(std::vector<uint32_t>& key, std::vector<uint32_t>& val) {
    const size_t n = key.size();
    uint32_t kmax = 0;
    bool sorted = true;
    for (size_t i = 0; i < n; ++i) {
        kmax = std::max(kmax, key[i]);
        sorted = sorted && (i == 0 || key[i - 1] <= key[i]);
    }
    if (sorted) return;
    constexpr int B = 11;
    constexpr uint32_t D = 1u << B, M = D - 1;
    const unsigned T = host_threads(n);
    std::vector<uint32_t> k2(n), v2(n);
    std::vector<size_t> cnt((size_t)T * D);
    for (int shift = 0; shift < 32 && (shift == 0 || (kmax >> shift) != 0); shift += B) {
        std::fill(cnt.begin(), cnt.end(), (size_t)0);
        parallel_chunks(n, T, [&](unsigned t, size_t lo, size_t hi) {
            size_t* c = cnt.data() + (size_t)t * D;
            for (size_t i = lo; i < hi; ++i) ++c[(key[i] >> shift) & M];
        });
        size_t run = 0;
        for (uint32_t d = 0; d < D; ++d)
            for (unsigned t = 0; t < T; ++t) {
                const size_t c = cnt[(size_t)t * D + d];
                cnt[(size_t)t * D + d] = run;
                run += c;
            }
        parallel_chunks(n, T, [&](unsigned t, size_t lo, size_t hi) {
            size_t* o = cnt.data() + (size_t)t * D;
            for (size_t i = lo; i < hi; ++i) {
                const size_t j = o[(key[i] >> shift) & M]++;
                k2[j] = key[i]; v2[j] = val[i];
            }
        });
        key.swap(k2); val.swap(v2);
    }
}

// Entries grouped by target: utarget ascending, off[g] .. off[g+1] the
// entries of group g in perm (the caller's order within a group).
inline void group_by(const std::vector<uint32_t>& tgt, std::vector<uint32_t>& utarget, std::vector<uint32_t>& off,
                     std::vector<uint32_t>& perm) {
    const uint32_t n = (uint32_t)tgt.size();
    std::vector<uint32_t> key(tgt);
    perm.resize(n);
    for (uint32_t i = 0; i < n; ++i) perm[i] = i;
    radix_sort_pairs(key, perm);
    utarget.clear();
    off.assign(1, 0);
    for (uint32_t i = 0; i < n; ++i) {
        if (i == 0 || key[i] != key[i - 1]) {
            if (i) off.push_back(i);
            utarget.push_back(key[i]);
        }
    }
    if (n) off.push_back(n);
}

}  // namespace efs_host
