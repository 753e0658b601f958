// Minimal stand-in for oneTBB's blocked_range, enough for the reference's CPU
// LBM solvers (src/aero/lbm3d/lbm3d_cpu.cpp:142, src/aero/lbm/lbm2d_cpu.cpp:220),
// which only read begin() and end().  Test infrastructure: used only to build
// the reference oracle under oracle/_ref.
#pragma once

#include <cstddef>

namespace tbb {

template <typename Value> class blocked_range {
public:
    blocked_range(Value begin, Value end) : begin_(begin), end_(end) {}
    [[nodiscard]] Value begin() const { return begin_; }
    [[nodiscard]] Value end() const { return end_; }
    [[nodiscard]] std::size_t size() const { return static_cast<std::size_t>(end_ - begin_); }
    [[nodiscard]] bool empty() const { return !(begin_ < end_); }

private:
    Value begin_;
    Value end_;
};

} // namespace tbb
