// CPU check of dig-appolo_b200/csrc/dsmc_hostpack.h: the threaded upload and
// download loops give, for every thread count, the same order, start
// offsets, values and bits as the serial loops they replace (restated here).
// Prints "ok" and exits 0, or names the first mismatch and exits 1.
#include "dsmc_hostpack.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

namespace hp = dsmc::hostpack;

namespace {

int failures = 0;

void check(bool ok, const char* what, int64_t n, int ncell, int threads)
{
    if (!ok && failures++ < 10) std::printf("mismatch: %s (n=%lld ncell=%d threads=%d)\n", what, (long long)n, ncell, threads);
}

// the serial upload loops: counting sort, then gather with conversion
void serial_order(int64_t n, const int32_t* cell, int ncell, std::vector<int>& st, std::vector<int64_t>& order)
{
    std::vector<int> cnt((size_t)ncell + 1, 0);
    for (int64_t i = 0; i < n; ++i) cnt[(size_t)cell[i] + 1]++;
    for (int c = 0; c < ncell; ++c) cnt[(size_t)c + 1] += cnt[(size_t)c];
    st.assign(cnt.begin(), cnt.end());
    order.assign((size_t)n, 0);
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int64_t i = 0; i < n; ++i) order[(size_t)fill[(size_t)cell[i]]++] = i;
}

template <class T>
bool same_bits(const std::vector<T>& a, const std::vector<T>& b)
{
    return a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), a.size() * sizeof(T)) == 0);
}

void run_case(int64_t n, int ncell, uint32_t seed, bool sorted_input)
{
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<int> pick(0, ncell - 1);
    std::normal_distribution<double> gauss(0.0, 3.0);
    std::vector<int32_t> cell((size_t)n);
    for (auto& c : cell) c = pick(rng);
    if (sorted_input) std::sort(cell.begin(), cell.end());
    std::vector<double> src((size_t)n), shift((size_t)ncell * 3);
    for (auto& s : src) s = gauss(rng) * 1e3;
    for (auto& s : shift) s = gauss(rng) * 1e3;

    std::vector<int> st0;
    std::vector<int64_t> ord0;
    serial_order(n, cell.data(), ncell, st0, ord0);
    std::vector<float> f0((size_t)n);
    std::vector<double> d0((size_t)n);
    std::vector<int32_t> c0((size_t)n);
    for (int64_t j = 0; j < n; ++j) {
        const int64_t i = ord0[(size_t)j];
        double v = src[(size_t)i];
        v = v - shift[(size_t)cell[(size_t)i] * 3 + 1];
        f0[(size_t)j] = (float)v;
        d0[(size_t)j] = src[(size_t)i];
        c0[(size_t)j] = cell[(size_t)i];
    }
    std::vector<double> w0((size_t)n);
    for (int64_t j = 0; j < n; ++j) w0[(size_t)j] = shift[(size_t)c0[(size_t)j] * 3 + 2] + (double)f0[(size_t)j];

    for (int threads : {1, 2, 3, 7, 16, hp::threads_for(n)}) {
        check(hp::cells_in_range(n, cell.data(), ncell, threads), "cells_in_range", n, ncell, threads);
        std::vector<int> st;
        std::vector<int64_t> ord;
        hp::order_by_cell(n, cell.data(), ncell, threads, st, ord);
        check(st == st0, "start", n, ncell, threads);
        check(ord == ord0, "order", n, ncell, threads);
        std::vector<float> f((size_t)n);
        hp::gather_convert<float>(n, ord.data(), src.data(), cell.data(), shift.data(), 1, f.data(), threads);
        check(same_bits(f, f0), "gather_convert<float> with shift", n, ncell, threads);
        std::vector<double> d((size_t)n);
        hp::gather_convert<double>(n, ord.data(), src.data(), cell.data(), nullptr, 0, d.data(), threads);
        check(same_bits(d, d0), "gather_convert<double>", n, ncell, threads);
        std::vector<int32_t> c((size_t)n);
        hp::gather_cells(n, ord.data(), cell.data(), c.data(), threads);
        check(c == c0, "gather_cells", n, ncell, threads);
        std::vector<double> w((size_t)n);
        hp::widen<float>(n, f.data(), c.data(), shift.data(), 2, w.data(), threads);
        check(same_bits(w, w0), "widen<float> with shift", n, ncell, threads);
        std::vector<double> wd((size_t)n);
        hp::widen<double>(n, d.data(), c.data(), nullptr, 0, wd.data(), threads);
        check(same_bits(wd, d0), "widen<double>", n, ncell, threads);
        if (n > 0) {
            std::vector<int32_t> bad(cell);
            bad[(size_t)(n - 1)] = ncell;                       // one id past the end, in the last chunk
            check(!hp::cells_in_range(n, bad.data(), ncell, threads), "cells_in_range rejects ncell", n, ncell, threads);
            bad[(size_t)(n - 1)] = cell[(size_t)(n - 1)];
            bad[0] = -1;
            check(!hp::cells_in_range(n, bad.data(), ncell, threads), "cells_in_range rejects -1", n, ncell, threads);
        }
    }
}

}  // namespace

int main()
{
    run_case(0, 5, 1, false);                  // no particles
    run_case(1, 1, 2, false);
    run_case(3, 10, 3, false);                 // fewer particles than threads
    run_case(1000, 37, 4, false);
    run_case(100000, 1, 5, false);             // one cell
    run_case(100000, 200000, 6, false);        // more cells than particles
    run_case((int64_t(1) << 20) + 17, 50000, 7, false);   // above the threading threshold
    run_case((int64_t(1) << 20) + 5, 3000, 8, true);      // already cell-major (a download fed back)
    if (failures) {
        std::printf("%d mismatches\n", failures);
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
