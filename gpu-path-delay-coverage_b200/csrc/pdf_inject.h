// pdf_inject.h -- host-side fault injection for tests of the error paths
// (pdf_test_inject): allocation calls of the library go through these
// wrappers, which fail as if memory were exhausted while an injected count
// for their kind is left.
#ifndef PDF_INJECT_H
#define PDF_INJECT_H

#include <cuda_runtime.h>

#include <cstddef>

// True (and one injected failure used up) when the next allocation of this
// kind (PDF_INJECT_*) must fail.
bool inject_fail(int site);
// cudaMalloc / cudaHostAlloc(cudaHostAllocDefault), or
// cudaErrorMemoryAllocation while a failure is injected.
cudaError_t dev_alloc(void **p, size_t bytes);
cudaError_t host_alloc(void **p, size_t bytes);

#endif
