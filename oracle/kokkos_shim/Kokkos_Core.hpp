// Kokkos-API shim over OpenMP — TEST INFRASTRUCTURE ONLY.
//
// This header is part of the oracle: it lets the reference's own headers
// (GraphKokkos include/matrix.h, include/matrix_la.h,
// include/betweenness_centrality.h) compile unmodified on a host that has no
// Kokkos installation, so that the reference algorithms can be run as the
// parity checker of the CUDA path.  It is never linked into the product
// library.
//
// It provides exactly the Kokkos names the reference uses (grep over the
// reference's include/ and src/):
//   View<T*> (label ctor zero-fills; operator()/operator[] const -> T&;
//   data(), size(), extent(0)), View<T*, scratch_memory_space, MemoryUnmanaged>
//   (ctor from a scratch handle + n, static shmem_size(n)), resize, deep_copy,
//   subview(View, pair), parallel_for (count / RangePolicy / TeamPolicy /
//   TeamThreadRange / ThreadVectorRange), parallel_reduce (count + Sum,
//   ThreadVectorRange + scalar), TeamPolicy::set_scratch_size + PerThread,
//   member_type (league_rank, team_size, thread_scratch), num_threads,
//   initialize/finalize, DefaultHostExecutionSpace, Experimental::equal,
//   KOKKOS_LAMBDA.
//
// Semantics chosen to match Kokkos where the reference depends on them:
//   * View copies are shallow and reference-counted (matrix.h:72-75 relies on it).
//   * resize() keeps the allocation when the extent is unchanged, otherwise
//     reallocates, zero-fills and copies the common prefix (Kokkos::resize).
//   * TeamPolicy runs one team per OpenMP thread with team size 1 and a
//     dynamic schedule over league ranks (Kokkos' OpenMP backend with
//     Kokkos::AUTO resolves to this on a host build).
//   * Per-thread scratch comes from a pool that each OpenMP thread keeps
//     between kernels (grown on demand, never shrunk), as Kokkos' scratch pool.
// Two documented deviations from Kokkos, both needed for the reference code
// to run as its author intended:
//   * Per-thread scratch is ZERO-FILLED for every team by default
//     (betweenness_centrality.h:347-363 and :379-397 read scratch before
//     writing it; real Kokkos leaves scratch uninitialised).  A caller that
//     times code which does not rely on it (the MSA product clears its
//     accumulator at the mask columns, matrix_la.h:614-616) turns the fill off
//     for a scope with kokkos_shim::ScratchZeroFill.
//   * deep_copy() between rank-1 views of different extents copies the common
//     prefix instead of aborting.  The reference k-truss loop
//     (main.cpp:106-130) passes a matrix whose Col extent is larger than its
//     nz into mxmm_msa (matrix_la.h:567), which real Kokkos rejects.
#pragma once

#include <omp.h>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>
#include <algorithm>

#define KOKKOS_LAMBDA [=]
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FUNCTION

namespace kokkos_shim {
// The calling OpenMP thread's scratch pool, at least `bytes` long.
inline char *thread_scratch(size_t bytes) {
    static thread_local std::vector<char> pool;
    if (pool.size() < bytes) {
        pool.clear();
        pool.shrink_to_fit();
        pool.resize(bytes);
    }
    return pool.data();
}
inline bool &zero_scratch_flag() {
    static bool zero = true;
    return zero;
}
// Scope in which TeamPolicy scratch is (or is not) zero-filled per team.
struct ScratchZeroFill {
    bool saved;
    explicit ScratchZeroFill(bool on) : saved(zero_scratch_flag()) { zero_scratch_flag() = on; }
    ~ScratchZeroFill() { zero_scratch_flag() = saved; }
};
}  // namespace kokkos_shim

namespace Kokkos {

inline void initialize(int &, char **) {}
inline void initialize() {}
inline void finalize() {}
inline int num_threads() { return omp_get_max_threads(); }

struct HostSpace {};
struct ScratchMemorySpace;
struct OpenMP {
    using scratch_memory_space = ScratchMemorySpace;
};
using DefaultExecutionSpace = OpenMP;
using DefaultHostExecutionSpace = OpenMP;
struct MemoryUnmanaged {};

// Per-thread scratch arena: bump allocation of consecutive chunks.
struct ScratchMemorySpace {
    char *base = nullptr;
    size_t capacity = 0;
    size_t offset = 0;
    void *get_shmem(size_t bytes) {
        size_t aligned = (offset + 7) & ~size_t(7);
        if (aligned + bytes > capacity) return nullptr;
        void *p = base + aligned;
        offset = aligned + bytes;
        return p;
    }
};

template <class DataType, class... Props>
class View;

// Managed (or unmanaged scratch) rank-1 view.
template <class T, class... Props>
class View<T *, Props...> {
public:
    using value_type = T;
    using pointer_type = T *;

    View() = default;
    View(const std::string &, size_t n) { allocate(n); }
    View(const char *, size_t n) { allocate(n); }
    // scratch view: bump-allocates n elements from a thread scratch handle
    View(ScratchMemorySpace &space, size_t n)
        : ptr_(static_cast<T *>(space.get_shmem(n * sizeof(T)))), n_(n) {}

    View(const View &) = default;
    View(View &&o) noexcept : hold_(std::move(o.hold_)), ptr_(o.ptr_), n_(o.n_) {
        o.ptr_ = nullptr;
        o.n_ = 0;
    }
    View &operator=(const View &) = default;
    View &operator=(View &&o) noexcept {
        if (this != &o) {
            hold_ = std::move(o.hold_);
            ptr_ = o.ptr_;
            n_ = o.n_;
            o.ptr_ = nullptr;
            o.n_ = 0;
        }
        return *this;
    }

    template <class I>
    T &operator()(I i) const { return ptr_[static_cast<size_t>(i)]; }
    template <class I>
    T &operator[](I i) const { return ptr_[static_cast<size_t>(i)]; }

    T *data() const { return ptr_; }
    size_t size() const { return n_; }
    size_t extent(int) const { return n_; }
    size_t span() const { return n_; }
    bool is_allocated() const { return ptr_ != nullptr; }

    static size_t shmem_size(size_t n) { return (n * sizeof(T) + 7) & ~size_t(7); }

    // shim internals
    void allocate(size_t n) {
        hold_ = std::shared_ptr<T[]>(new T[n > 0 ? n : 1]());
        ptr_ = hold_.get();
        n_ = n;
    }
    View sub(size_t b, size_t e) const {
        View v(*this);
        v.ptr_ = ptr_ + b;
        v.n_ = e - b;
        return v;
    }

private:
    std::shared_ptr<T[]> hold_;
    T *ptr_ = nullptr;
    size_t n_ = 0;
};

template <class T, class... P>
void resize(View<T *, P...> &v, size_t n) {
    if (v.size() == n && (v.data() != nullptr || n == 0)) return;
    View<T *, P...> nv("", n);
    size_t common = std::min(n, v.size());
    if (common) std::memcpy(static_cast<void *>(nv.data()), v.data(), common * sizeof(T));
    v = nv;
}

template <class T, class... P, class U, class... Q>
void deep_copy(const View<T *, P...> &dst, const View<U *, Q...> &src) {
    size_t common = std::min(dst.size(), src.size());
    if (common == 0 || static_cast<const void *>(dst.data()) == static_cast<const void *>(src.data()))
        return;
    std::memmove(static_cast<void *>(dst.data()), src.data(), common * sizeof(T));
}

template <class T, class... P>
void deep_copy(const View<T *, P...> &dst, const T &value) {
    for (size_t i = 0; i < dst.size(); ++i) dst(i) = value;
}

template <class T, class... P, class I>
View<T *, P...> subview(const View<T *, P...> &v, std::pair<I, I> r) {
    return v.sub(static_cast<size_t>(r.first), static_cast<size_t>(r.second));
}

template <class T, class... P>
void swap(View<T *, P...> &a, View<T *, P...> &b) {
    View<T *, P...> t(std::move(a));
    a = std::move(b);
    b = std::move(t);
}

// ----- policies -----------------------------------------------------------
struct Dynamic {};
struct Static {};
template <class S>
struct Schedule {};
struct ChunkSize {
    explicit ChunkSize(int c) : value(c) {}
    int value;
};
struct AUTO_t {};
constexpr AUTO_t AUTO{};

template <class... Args>
struct RangePolicy {
    RangePolicy(int64_t b, int64_t e) : begin(b), end(e) {}
    RangePolicy(int64_t b, int64_t e, ChunkSize c) : begin(b), end(e), chunk(c.value) {}
    int64_t begin, end;
    int chunk = 0;
};

struct PerThreadValue {
    size_t bytes;
};
inline PerThreadValue PerThread(size_t bytes) { return PerThreadValue{bytes}; }

class TeamMember {
public:
    TeamMember(int rank, int league, ScratchMemorySpace *scratch)
        : rank_(rank), league_(league), scratch_(scratch) {}
    int league_rank() const { return rank_; }
    int league_size() const { return league_; }
    int team_rank() const { return 0; }
    int team_size() const { return 1; }
    ScratchMemorySpace &thread_scratch(int) const { return *scratch_; }
    ScratchMemorySpace &team_scratch(int) const { return *scratch_; }
    void team_barrier() const {}

private:
    int rank_, league_;
    ScratchMemorySpace *scratch_;
};

template <class... Args>
struct TeamPolicy {
    using member_type = TeamMember;
    TeamPolicy() = default;
    TeamPolicy(int64_t league, AUTO_t) : league_size(league) {}
    TeamPolicy(int64_t league, AUTO_t, int) : league_size(league) {}
    TeamPolicy(int64_t league, int) : league_size(league) {}
    TeamPolicy(int64_t league, int, int) : league_size(league) {}
    template <class... Other>
    TeamPolicy(const TeamPolicy<Other...> &o)
        : league_size(o.league_size), scratch_bytes(o.scratch_bytes) {}
    TeamPolicy set_scratch_size(int, PerThreadValue v) const {
        TeamPolicy p(*this);
        p.scratch_bytes = v.bytes;
        return p;
    }
    int64_t league_size = 0;
    size_t scratch_bytes = 0;
};

template <class M>
struct TeamThreadRangeBoundaries {
    int64_t begin, end;
};
template <class I1, class I2>
TeamThreadRangeBoundaries<TeamMember> TeamThreadRange(const TeamMember &, I1 b, I2 e) {
    return {static_cast<int64_t>(b), static_cast<int64_t>(e)};
}
template <class M>
struct ThreadVectorRangeBoundaries {
    int64_t begin, end;
};
template <class I1, class I2>
ThreadVectorRangeBoundaries<TeamMember> ThreadVectorRange(const TeamMember &, I1 b, I2 e) {
    return {static_cast<int64_t>(b), static_cast<int64_t>(e)};
}
template <class I1>
ThreadVectorRangeBoundaries<TeamMember> ThreadVectorRange(const TeamMember &, I1 e) {
    return {0, static_cast<int64_t>(e)};
}

// ----- parallel_for ---------------------------------------------------------
template <class F>
void parallel_for(const std::string &, size_t n, const F &f) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) f(i);
}
template <class F, class... A>
void parallel_for(const std::string &, const RangePolicy<A...> &p, const F &f) {
    const int chunk = p.chunk > 0 ? p.chunk : 1;
#pragma omp parallel for schedule(dynamic, chunk)
    for (int64_t i = p.begin; i < p.end; ++i) f(i);
}
template <class F, class... A>
void parallel_for(const std::string &, const TeamPolicy<A...> &p, const F &f) {
    const size_t bytes = p.scratch_bytes;
    const int64_t league = p.league_size;
    const bool zero = kokkos_shim::zero_scratch_flag();
#pragma omp parallel
    {
        char *arena = kokkos_shim::thread_scratch(bytes > 0 ? bytes : 8);
#pragma omp for schedule(dynamic, 1)
        for (int64_t r = 0; r < league; ++r) {
            if (zero) std::memset(arena, 0, bytes);
            ScratchMemorySpace space{arena, bytes, 0};
            TeamMember member(static_cast<int>(r), static_cast<int>(league), &space);
            f(member);
        }
    }
}
template <class F>
void parallel_for(const TeamThreadRangeBoundaries<TeamMember> &r, const F &f) {
    for (int64_t i = r.begin; i < r.end; ++i) f(static_cast<int>(i));
}
template <class F>
void parallel_for(const ThreadVectorRangeBoundaries<TeamMember> &r, const F &f) {
    for (int64_t i = r.begin; i < r.end; ++i) f(static_cast<int>(i));
}

// ----- parallel_reduce ------------------------------------------------------
template <class T>
struct Sum {
    explicit Sum(T &r) : ref(r) {}
    T &ref;
};
template <class F, class T>
void parallel_reduce(const std::string &, size_t n, const F &f, Sum<T> s) {
    T total = T(0);
#pragma omp parallel
    {
        T local = T(0);
#pragma omp for schedule(static) nowait
        for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) f(i, local);
#pragma omp critical
        total += local;
    }
    s.ref = total;
}
template <class F, class T>
void parallel_reduce(const ThreadVectorRangeBoundaries<TeamMember> &r, const F &f, T &result) {
    T acc = T(0);
    for (int64_t i = r.begin; i < r.end; ++i) f(static_cast<int>(i), acc);
    result = acc;
}

inline void fence() {}

namespace Experimental {
template <class Exec, class T, class... P, class U, class... Q>
bool equal(const Exec &, const View<T *, P...> &a, const View<U *, Q...> &b) {
    if (a.size() != b.size()) return false;
    for (size_t i = 0; i < a.size(); ++i)
        if (!(a(i) == b(i))) return false;
    return true;
}
}  // namespace Experimental

}  // namespace Kokkos
