// CPU checks of the engine's host planning helpers (efs_b200/csrc/efs_host.h):
// the threaded radix sort equals std::stable_sort by key (values in input
// order within equal keys), group_by's groups, and parallel_chunks covers
// [0, n) exactly once.  Prints "ok" or the first failure; exit code 0 / 1.
#include "efs_host.h"

#include <atomic>
#include <cstdio>
#include <random>
#include <utility>

static int fail(const char* what, size_t n, int kind) {
    std::printf("FAIL %s n=%zu kind=%d\n", what, n, kind);
    return 1;
}

int main() {
    std::mt19937 rng(7);
    const size_t sizes[] = {0, 1, 2, 5, 1000, 65535, 65536, 70001, 300001, 2031616};
    for (size_t n : sizes) {
        for (int kind = 0; kind < 5; ++kind) {
            std::vector<uint32_t> k(n), v(n);
            for (size_t i = 0; i < n; ++i) {
                switch (kind) {
                    case 0: k[i] = rng() % 1000; break;                        // many repeats
                    case 1: k[i] = rng(); break;                               // full 32-bit keys
                    case 2: k[i] = (uint32_t)(i / 3); break;                   // already sorted
                    case 3: k[i] = (uint32_t)(n - i); break;                   // reversed
                    default: k[i] = (uint32_t)((i * 2654435761u) % 402653184u);  // field-index range
                }
                v[i] = (uint32_t)i;
            }
            std::vector<std::pair<uint32_t, uint32_t>> ref(n);
            for (size_t i = 0; i < n; ++i) ref[i] = {k[i], v[i]};
            std::stable_sort(ref.begin(), ref.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
            std::vector<uint32_t> tgt(k);
            efs_host::radix_sort_pairs(k, v);
            for (size_t i = 0; i < n; ++i)
                if (k[i] != ref[i].first || v[i] != ref[i].second) return fail("radix_sort_pairs", n, kind);
            std::vector<uint32_t> ut, off, perm;
            efs_host::group_by(tgt, ut, off, perm);
            if (off.size() != ut.size() + 1 || off.back() != n || off[0] != 0)
                return fail("group_by offsets", n, kind);
            for (size_t g = 0; g < ut.size(); ++g) {
                if (g && ut[g] <= ut[g - 1]) return fail("group_by order", n, kind);
                for (uint32_t j = off[g]; j < off[g + 1]; ++j) {
                    if (tgt[perm[j]] != ut[g]) return fail("group_by member", n, kind);
                    if (j > off[g] && perm[j] <= perm[j - 1]) return fail("group_by stability", n, kind);
                }
            }
        }
        for (unsigned T : {1u, 2u, 3u, 16u}) {
            std::vector<std::atomic<int>> hits(n);
            for (auto& h : hits) h = 0;
            efs_host::parallel_chunks(n, T, [&](unsigned, size_t lo, size_t hi) {
                for (size_t i = lo; i < hi; ++i) hits[i]++;
            });
            for (size_t i = 0; i < n; ++i)
                if (hits[i] != 1) return fail("parallel_chunks", n, (int)T);
        }
    }
    if (efs_host::host_threads(1000) != 1 || efs_host::host_threads(1u << 20) < 1 || efs_host::host_threads(1u << 20) > 16)
        return fail("host_threads", 0, 0);
    std::printf("ok\n");
    return 0;
}
