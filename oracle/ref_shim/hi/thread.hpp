// Stand-in for <hi/thread.hpp> (Win32 thread wrappers).  The oracle drives the
// reference's estimator from its own harness threads, so nothing is needed here.
#pragma once
#include <hi/lang.hpp>
namespace hi {
// Base of the reference's integrator threads (libhi/hi/thread/thread.hpp):
// the oracle never starts them; run() is called directly where needed.
class thread {
 public:
  virtual ~thread() {}
  virtual void run() = 0;
  void start() { run(); }
  void join() {}
};
}  // namespace hi
