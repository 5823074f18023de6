// devmem.h - the library's one path to device memory.
//
// Every device allocation and free of the library goes through dev_alloc and
// dev_free.  They keep a count of live allocations, and dev_alloc can be told
// to fail the n-th call from now (ae_debug_fail_alloc_after): that is how the
// out-of-memory paths of ae_create, ae_prepare_fast, ae_serve_create and the
// rest are exercised without exhausting a real GPU.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

namespace ae {
cudaError_t dev_alloc(void **p, size_t bytes);
void dev_free(void *p);
// Status of the last ae_create / ae_serve_create on the calling thread.
void set_create_status(int status);
int create_status();
}  // namespace ae
