// Oracle test infrastructure: stand-in for Cubism's Profiler as used by
// SimulationData::startProfiler/stopProfiler (SimulationData.cpp:187-205).
// Accumulates wall time per named region so the CPU baseline can report the
// per-stage times of the reference's own operators.
#pragma once
#include <chrono>
#include <map>
#include <string>
#include <vector>
namespace cubism {
class Profiler
{
  using clock = std::chrono::steady_clock;
  std::vector<std::pair<std::string, clock::time_point>> stack;
 public:
  std::map<std::string, double> seconds;
  std::map<std::string, long> calls;
  void push_start(const std::string& name) { stack.push_back({name, clock::now()}); }
  void pop_stop() {
    if (stack.empty()) return;
    const auto e = clock::now();
    const auto& top = stack.back();
    seconds[top.first] += std::chrono::duration<double>(e - top.second).count();
    calls[top.first] += 1;
    stack.pop_back();
  }
  std::string currentAgentName() const { return stack.empty() ? "" : stack.back().first; }
  void printSummary() const {}
  void reset() {}
};
}
