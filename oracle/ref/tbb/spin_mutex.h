// No-op stand-in for tbb::spin_mutex (single-threaded parity checker).
#pragma once
namespace tbb { struct spin_mutex { struct scoped_lock { scoped_lock() {} explicit scoped_lock(spin_mutex&) {} void acquire(spin_mutex&) {} void release() {} }; }; }
