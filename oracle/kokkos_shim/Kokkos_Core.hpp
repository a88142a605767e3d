// Kokkos_Core.hpp -- project-written host shim of the small Kokkos API subset
// that the HOW-MHD reference sources use. TEST INFRASTRUCTURE ONLY: it exists so
// that the reference's own src/*.cpp compile unmodified into the CPU oracle
// under oracle/_ref/. Nothing in the product links it.
//
// Written from the public semantics of the Kokkos API (Kokkos itself is not
// installed here and nothing is copied from it):
//   * View<double*...*> : rank 1..5, LayoutRight (last index fastest),
//     zero-initialised on construction, shallow reference-counted copies,
//     operator() const returning a mutable reference.
//   * RangePolicy<>, MDRangePolicy<Rank<N>> with {begin} / {end} arrays.
//   * parallel_for / parallel_reduce (Max<double> reducers), fence,
//     deep_copy, create_mirror_view[_and_copy], atomic_add.
// Parallelisation: OpenMP over the outermost index (the two outermost for
// rank >= 3).  The innermost index always runs serially and in order, which
// keeps the reference's atomic_add over the characteristic index m
// (ssprk.cpp:941-943) deterministic and ordered m = 0..6.
//
// Optional per-label wall-clock timers: set HOW_REF_TIMERS=1 and the totals
// are printed to stderr at exit (the CPU time split of the reference path).
#pragma once

#include <array>
#include <algorithm>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <utility>
#include <vector>
#include <cstdio>
#include <omp.h>

#define KOKKOS_LAMBDA [=]
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FUNCTION

namespace Kokkos {

struct HostSpace {};

namespace impl {

template <class T> struct rank_of { static constexpr int value = 0; using scalar = T; };
template <class T> struct rank_of<T*> {
    static constexpr int value = rank_of<T>::value + 1;
    using scalar = typename rank_of<T>::scalar;
};

struct LabelTimers {
    bool on = false;
    std::map<std::string, double> total;
    LabelTimers() {
        const char* e = std::getenv("HOW_REF_TIMERS");
        on = (e != nullptr && e[0] == '1');
    }
    ~LabelTimers() {
        if (!on) return;
        std::vector<std::pair<double, std::string>> v;
        double sum = 0.0;
        for (auto& kv : total) { v.push_back({kv.second, kv.first}); sum += kv.second; }
        std::sort(v.rbegin(), v.rend());
        std::fprintf(stderr, "[ref-timers] total %.4f s\n", sum);
        for (auto& p : v)
            std::fprintf(stderr, "[ref-timers] %-40s %10.4f s %6.2f %%\n",
                         p.second.c_str(), p.first, sum > 0 ? 100.0 * p.first / sum : 0.0);
    }
};
inline LabelTimers& timers() { static LabelTimers t; return t; }

struct ScopedLabel {
    const std::string* label; double t0;
    explicit ScopedLabel(const std::string& l) : label(&l), t0(timers().on ? omp_get_wtime() : 0.0) {}
    ~ScopedLabel() { if (timers().on) timers().total[*label] += omp_get_wtime() - t0; }
};

} // namespace impl

template <class DataType>
class View {
public:
    static constexpr int rank = impl::rank_of<DataType>::value;
    using value_type = typename impl::rank_of<DataType>::scalar;
    static_assert(rank >= 1 && rank <= 5, "shim supports rank 1..5");

    View() = default;

    View(const std::string& label, std::size_t n0, std::size_t n1 = 1, std::size_t n2 = 1,
         std::size_t n3 = 1, std::size_t n4 = 1)
        : label_(label) {
        const std::size_t n[5] = {n0, n1, n2, n3, n4};
        std::size_t total = 1;
        for (int r = 0; r < 5; ++r) { ext_[r] = (r < rank) ? n[r] : 1; }
        for (int r = 0; r < rank; ++r) total *= ext_[r];
        // strides, LayoutRight
        std::size_t s = 1;
        for (int r = rank - 1; r >= 0; --r) { stride_[r] = s; s *= ext_[r]; }
        store_ = std::make_shared<std::vector<value_type>>(total, value_type(0));
        ptr_ = store_->data();
        size_ = total;
    }

    value_type& operator()(long i0) const { return ptr_[i0]; }
    value_type& operator()(long i0, long i1) const {
        return ptr_[i0 * stride_[0] + i1];
    }
    value_type& operator()(long i0, long i1, long i2) const {
        return ptr_[i0 * stride_[0] + i1 * stride_[1] + i2];
    }
    value_type& operator()(long i0, long i1, long i2, long i3) const {
        return ptr_[i0 * stride_[0] + i1 * stride_[1] + i2 * stride_[2] + i3];
    }
    value_type& operator()(long i0, long i1, long i2, long i3, long i4) const {
        return ptr_[i0 * stride_[0] + i1 * stride_[1] + i2 * stride_[2] + i3 * stride_[3] + i4];
    }

    std::size_t extent(int r) const { return ext_[r]; }
    std::size_t size() const { return size_; }
    value_type* data() const { return ptr_; }
    const std::string& label() const { return label_; }

private:
    std::string label_;
    std::shared_ptr<std::vector<value_type>> store_;
    value_type* ptr_ = nullptr;
    std::size_t size_ = 0;
    std::size_t ext_[5] = {1, 1, 1, 1, 1};
    std::size_t stride_[5] = {1, 1, 1, 1, 1};
};

template <int N> struct Rank { static constexpr int value = N; };

template <class... Args>
struct RangePolicy {
    long b, e;
    RangePolicy(long b_, long e_) : b(b_), e(e_) {}
};

template <class R>
struct MDRangePolicy {
    static constexpr int N = R::value;
    std::array<long, N> lo, hi;
    MDRangePolicy(const std::array<long, N>& l, const std::array<long, N>& h) : lo(l), hi(h) {}
};

template <class T>
struct Max {
    T& ref;
    explicit Max(T& r) : ref(r) {}
};

inline void fence() {}
inline void initialize(int&, char**) {}
inline void initialize() {}
inline void finalize() {}

inline void atomic_add(double* p, double v) {
#pragma omp atomic
    *p += v;
}

// ---------------------------------------------------------------- parallel_for
template <class F>
void parallel_for(const std::string& label, const RangePolicy<>& p, const F& f) {
    impl::ScopedLabel t(label);
#pragma omp parallel for schedule(static)
    for (long i = p.b; i < p.e; ++i) f((int)i);
}

template <class F>
void parallel_for(const std::string& label, long n, const F& f) {
    parallel_for(label, RangePolicy<>(0, n), f);
}

template <class F>
void parallel_for(const std::string& label, const MDRangePolicy<Rank<2>>& p, const F& f) {
    impl::ScopedLabel t(label);
#pragma omp parallel for schedule(static)
    for (long i = p.lo[0]; i < p.hi[0]; ++i)
        for (long j = p.lo[1]; j < p.hi[1]; ++j) f((int)i, (int)j);
}

template <class F>
void parallel_for(const std::string& label, const MDRangePolicy<Rank<3>>& p, const F& f) {
    impl::ScopedLabel t(label);
#pragma omp parallel for collapse(2) schedule(static)
    for (long i = p.lo[0]; i < p.hi[0]; ++i)
        for (long j = p.lo[1]; j < p.hi[1]; ++j)
            for (long k = p.lo[2]; k < p.hi[2]; ++k) f((int)i, (int)j, (int)k);
}

template <class F>
void parallel_for(const std::string& label, const MDRangePolicy<Rank<4>>& p, const F& f) {
    impl::ScopedLabel t(label);
#pragma omp parallel for collapse(2) schedule(static)
    for (long i = p.lo[0]; i < p.hi[0]; ++i)
        for (long j = p.lo[1]; j < p.hi[1]; ++j)
            for (long k = p.lo[2]; k < p.hi[2]; ++k)
                for (long l = p.lo[3]; l < p.hi[3]; ++l) f((int)i, (int)j, (int)k, (int)l);
}

// ------------------------------------------------------------- parallel_reduce
// Only the form used by the reference: a rank-3 MDRange with three Max reducers
// (tstep.cpp:28-83).  max is exact, so the combine order does not matter.
template <class F>
void parallel_reduce(const std::string& label, const MDRangePolicy<Rank<3>>& p, const F& f,
                     Max<double> r0, Max<double> r1, Max<double> r2) {
    impl::ScopedLabel t(label);
    const double lowest = -1.7976931348623157e308;
    double g0 = lowest, g1 = lowest, g2 = lowest;
#pragma omp parallel
    {
        double a = lowest, b = lowest, c = lowest;
#pragma omp for collapse(2) schedule(static)
        for (long i = p.lo[0]; i < p.hi[0]; ++i)
            for (long j = p.lo[1]; j < p.hi[1]; ++j)
                for (long k = p.lo[2]; k < p.hi[2]; ++k) f((int)i, (int)j, (int)k, a, b, c);
#pragma omp critical
        {
            g0 = std::max(g0, a); g1 = std::max(g1, b); g2 = std::max(g2, c);
        }
    }
    r0.ref = g0; r1.ref = g1; r2.ref = g2;
}

// ------------------------------------------------------------------ deep_copy
template <class D>
void deep_copy(const View<D>& v, typename View<D>::value_type x) {
    auto* p = v.data();
    const long n = (long)v.size();
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) p[i] = x;
}

template <class D1, class D2>
void deep_copy(const View<D1>& dst, const View<D2>& src) {
    const long n = (long)std::min(dst.size(), src.size());
    auto* d = dst.data();
    auto* s = src.data();
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) d[i] = s[i];
}

// Host views are their own mirrors.
template <class D> View<D> create_mirror_view(const View<D>& v) { return v; }
template <class D> View<D> create_mirror_view(const HostSpace&, const View<D>& v) { return v; }
template <class D> View<D> create_mirror_view_and_copy(const HostSpace&, const View<D>& v) { return v; }

} // namespace Kokkos
