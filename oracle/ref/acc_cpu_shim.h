// Pre-include shim for compiling the reference's CPU (ALTCPU) E-step kernels
// (src/acc/cpu/cpu_kernels/*.h) outside its CMake build, as a parity checker.
// The kernels only name these GPU-build types and host allocators; nothing
// here is called by the code paths the wrapper uses.  Test infrastructure.
#pragma once
#include <cstddef>
#include <cstdlib>
#include <limits>
int pin_alloc(void** ptr, size_t size);
void pin_free(void* ptr);
class CudaAllocatorTask {
public:
    unsigned char* alloc(size_t) { return nullptr; }
    void free(unsigned char*, size_t) {}
};
class CudaAllocatorThread {
public:
    bool canAdd(size_t, int) { return true; }
    CudaAllocatorTask* addOneTask(int, size_t) { return nullptr; }
    void freeOneTask(CudaAllocatorTask*) {}
};
