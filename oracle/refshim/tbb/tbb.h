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

template <typename Range, typename Body>
void parallel_for(const Range& range, const Body& body) {
    body(range);
}

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
