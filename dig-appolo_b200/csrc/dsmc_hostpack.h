// Host-side loops of the particle upload and download (dsmc_upload_particles,
// dsmc_download_particles), split over threads for large particle counts.
// Plain C++17, no CUDA: the same header builds into a CPU test.
//
// The order is the library's canonical one: cell-major, and within a cell
// the input order (a stable counting sort by cell). Conversions are the
// single expressions of the serial loops they replace, so every thread count
// gives the same bits.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace dsmc {
namespace hostpack {

// Threads for n particles: one below 2^20 (thread start-up would dominate),
// else the hardware's, at most 16.
inline int threads_for(int64_t n)
{
    if (n < (int64_t(1) << 20)) return 1;
    const unsigned hw = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(hw == 0 ? 1u : hw, 16u));
}

// f(begin, end, t) over nthreads contiguous chunks of [0, n), chunk t on
// thread t (chunk 0 on the calling thread). Chunks write disjoint outputs,
// so a chunk whose thread cannot be started runs on the calling thread.
template <class F>
void parallel_for(int64_t n, int nthreads, F f)
{
    nthreads = std::max(1, nthreads);
    if (nthreads == 1 || n < nthreads) {
        f(int64_t(0), n, 0);
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve((size_t)nthreads - 1);
    const int64_t step = (n + nthreads - 1) / nthreads;
    for (int t = 1; t < nthreads; ++t) {
        const int64_t b = std::min(n, step * t), e = std::min(n, step * (t + 1));
        try {
            pool.emplace_back([=, &f] { f(b, e, t); });
        } catch (...) {
            f(b, e, t);
        }
    }
    f(int64_t(0), std::min(n, step), 0);
    for (auto& th : pool) th.join();
}

// Whether every cell id lies in [0, ncell).
inline bool cells_in_range(int64_t n, const int32_t* cell, int ncell, int nthreads)
{
    std::atomic<bool> ok{true};
    parallel_for(n, nthreads, [&](int64_t b, int64_t e, int) {
        for (int64_t i = b; i < e; ++i)
            if (cell[i] < 0 || cell[i] >= ncell) {
                ok.store(false, std::memory_order_relaxed);
                return;
            }
    });
    return ok.load();
}

// Stable counting sort by cell: start[c] is the first slot of cell c
// (start[ncell] = n) and order[j] the input index that slot j holds. Cells
// must be in range (cells_in_range).
inline void order_by_cell(int64_t n, const int32_t* cell, int ncell, int nthreads, std::vector<int>& start,
                          std::vector<int64_t>& order)
{
    nthreads = std::max(1, (int)std::min<int64_t>(nthreads, std::max<int64_t>(n, 1)));
    start.assign((size_t)ncell + 1, 0);
    order.resize((size_t)n);
    // per-chunk histograms, chunk t = the t-th contiguous input range
    std::vector<std::vector<int>> hist((size_t)nthreads);
    parallel_for(n, nthreads, [&](int64_t b, int64_t e, int t) {
        std::vector<int>& h = hist[(size_t)t];
        h.assign((size_t)ncell, 0);
        for (int64_t i = b; i < e; ++i) h[(size_t)cell[i]]++;
    });
    for (auto& h : hist)
        if (h.empty()) h.assign((size_t)ncell, 0);
    // slots: cells in order, within a cell the chunks in input order
    int run = 0;
    for (int c = 0; c < ncell; ++c) {
        start[(size_t)c] = run;
        for (int t = 0; t < nthreads; ++t) {
            const int k = hist[(size_t)t][(size_t)c];
            hist[(size_t)t][(size_t)c] = run;
            run += k;
        }
    }
    start[(size_t)ncell] = run;
    parallel_for(n, nthreads, [&](int64_t b, int64_t e, int t) {
        std::vector<int>& next = hist[(size_t)t];
        for (int64_t i = b; i < e; ++i) order[(size_t)next[(size_t)cell[i]]++] = i;
    });
}

// dst[j] = (Out)(src[i] - shift[cell[i] * 3 + comp]) with i = order[j]; no
// shift when shift is null.
template <class Out>
void gather_convert(int64_t n, const int64_t* order, const double* src, const int32_t* cell, const double* shift,
                    int comp, Out* dst, int nthreads)
{
    parallel_for(n, nthreads, [&](int64_t b, int64_t e, int) {
        for (int64_t j = b; j < e; ++j) {
            const int64_t i = order[j];
            double v = src[i];
            if (shift) v = v - shift[(size_t)cell[i] * 3 + comp];
            dst[j] = (Out)v;
        }
    });
}

// dst[j] = cell[order[j]]
inline void gather_cells(int64_t n, const int64_t* order, const int32_t* cell, int32_t* dst, int nthreads)
{
    parallel_for(n, nthreads, [&](int64_t b, int64_t e, int) {
        for (int64_t j = b; j < e; ++j) dst[j] = cell[order[j]];
    });
}

// dst[j] = shift[cell[j] * 3 + comp] + (double)src[j]; no shift when shift is null.
template <class In>
void widen(int64_t n, const In* src, const int32_t* cell, const double* shift, int comp, double* dst, int nthreads)
{
    parallel_for(n, nthreads, [&](int64_t b, int64_t e, int) {
        for (int64_t j = b; j < e; ++j) {
            double v = (double)src[j];
            if (shift) v = shift[(size_t)cell[j] * 3 + comp] + v;
            dst[j] = v;
        }
    });
}

// memcpy split over threads (byte ranges; every thread count gives the same
// bytes)
inline void parallel_copy(void* dst, const void* src, size_t bytes, int nthreads)
{
    char* d = static_cast<char*>(dst);
    const char* s = static_cast<const char*>(src);
    parallel_for((int64_t)bytes, nthreads, [&](int64_t b, int64_t e, int) {
        if (e > b) std::memcpy(d + b, s + b, (size_t)(e - b));
    });
}

}  // namespace hostpack
}  // namespace dsmc
