// bg_build.cu -- native construction helpers (host code).
//
// bg_fixed_indegree_csr: the connectivity of random_matrix_fixed_column
// (construction.py:149-177): every target receives exactly k distinct
// sources drawn uniformly, returned as CSR rows over sources with ascending
// targets.  Draws are a pure function of (seed, target, attempt), so the
// result does not depend on the number of worker threads.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "bg_common.cuh"
#include "../../include/brian_b200.h"

extern "C" BG_API int bg_fixed_indegree_csr(int64_t n_src, int64_t n_tgt, int64_t k, uint64_t seed,
                                             int64_t *rowptr, int32_t *cols) {
    if (n_src <= 0 || n_tgt < 0 || k < 0 || k > n_src || !rowptr || (n_tgt * k > 0 && !cols)) return BG_EINVAL;
    if (n_src > INT32_MAX || n_tgt > INT32_MAX) return BG_EINVAL;
    const int64_t nnz = n_tgt * k;
    std::vector<int32_t> src((size_t)nnz);
    unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    auto work = [&](int64_t j0, int64_t j1) {
        std::vector<int32_t> buf;
        for (int64_t j = j0; j < j1; ++j) {
            int32_t *s = src.data() + j * k;
            int64_t have = 0; uint64_t attempt = 0;
            while (have < k) {
                // draw the missing ones, then sort and drop duplicates
                for (int64_t r = have; r < k; r += 2) {
                    uint32_t c[4] = {(uint32_t)j, (uint32_t)((uint64_t)j >> 32), (uint32_t)attempt, (uint32_t)(attempt >> 32)};
                    bg_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
                    ++attempt;
                    s[r] = (int32_t)(((uint64_t)c[0] * (uint64_t)n_src) >> 32);
                    if (r + 1 < k) s[r + 1] = (int32_t)(((uint64_t)c[1] * (uint64_t)n_src) >> 32);
                }
                std::sort(s, s + k);
                have = std::unique(s, s + k) - s;
            }
        }
    };
    std::vector<std::thread> th;
    const int64_t per = (n_tgt + nth - 1) / nth;
    for (unsigned t = 0; t < nth; ++t) {
        int64_t j0 = t * per, j1 = std::min<int64_t>(n_tgt, j0 + per);
        if (j0 < j1) th.emplace_back(work, j0, j1);
    }
    for (auto &t : th) t.join();
    // counting sort by source, stable in target order -> ascending columns
    std::memset(rowptr, 0, sizeof(int64_t) * (size_t)(n_src + 1));
    for (int64_t p = 0; p < nnz; ++p) rowptr[src[p] + 1]++;
    for (int64_t i = 0; i < n_src; ++i) rowptr[i + 1] += rowptr[i];
    std::vector<int64_t> fill(rowptr, rowptr + n_src);
    for (int64_t j = 0; j < n_tgt; ++j) {
        const int32_t *s = src.data() + j * k;
        for (int64_t r = 0; r < k; ++r) cols[fill[s[r]]++] = (int32_t)j;
    }
    return BG_OK;
}
