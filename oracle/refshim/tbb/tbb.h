// TEST INFRASTRUCTURE ONLY: serial stand-in for the Intel TBB interfaces that betajippity/Ariel's
// FLIP step includes (`#include <tbb/tbb.h>`, e.g. src/sim/flip.hpp:10).  TBB only schedules the
// work; it computes nothing.  `parallel_for` hands the whole range to the body in one call, so
// every loop runs in ascending index order on one thread.  That is the deterministic serial
// order in which the oracle resolves the reference's benign races (BuildPreconditioner and
// ApplyPreconditioner read neighbours that other TBB workers write, src/sim/solver.inl:104-286).
#ifndef ARIEL_REFSHIM_TBB_H
#define ARIEL_REFSHIM_TBB_H

#include <cstddef>
#include <vector>
#if defined(ARIEL_TBB_OPENMP) && defined(_OPENMP)
#include <omp.h>
#endif

namespace tbb {

template <typename Value>
class blocked_range {
  public:
    blocked_range(Value begin, Value end) : m_begin(begin), m_end(end) {}
    Value begin() const { return m_begin; }
    Value end() const { return m_end; }
    bool empty() const { return !(m_begin < m_end); }

  private:
    Value m_begin, m_end;
};

#if defined(ARIEL_TBB_OPENMP) && defined(_OPENMP)
// Timing build (oracle/_ref/libariel_reference_omp.so, the benchmark's CPU reference arm): the
// range is cut into one contiguous piece per OpenMP thread, each handed to the body, as TBB's
// scheduler would cut it across its workers.  The reference's benign races then run as races,
// as they do under TBB; this build is timed, never compared.
template <typename Range, typename Body>
void parallel_for(const Range& range, const Body& body) {
    typedef decltype(range.begin()) V;
    const long long b = (long long)range.begin(), e = (long long)range.end();
    const long long len = e - b;
    if (len <= 1 || omp_in_parallel()) {
        body(range);
        return;
    }
#pragma omp parallel
    {
        const long long nt = omp_get_num_threads(), t = omp_get_thread_num();
        const long long lo = b + len * t / nt, hi = b + len * (t + 1) / nt;
        if (lo < hi) body(Range((V)lo, (V)hi));
    }
}
#else
template <typename Range, typename Body>
void parallel_for(const Range& range, const Body& body) {
    body(range);
}
#endif

class task {
  public:
    virtual ~task() {}
    virtual task* execute() = 0;
};

class mutex {
  public:
    void lock() {}
    void unlock() {}
};

template <typename T>
class concurrent_vector : public std::vector<T> {};

}  // namespace tbb

#endif
