// The fixed device scratch of pw_afd_noalloc.  It lives in its own
// translation unit, so under lazy module loading (CUDA_MODULE_LOADING=LAZY,
// the default since CUDA 12.2) its module, and the array with it, is loaded
// only by the first call that asks for its address, not by the library's
// other entry points; under EAGER loading every context that loads the
// library reserves it.  Every device gets its own copy of the array in its
// context.
#include "pw_common.cuh"

namespace pw {

static __device__ __align__(256) unsigned char noalloc_scratch_bytes[PW_NOALLOC_SCRATCH_BYTES];

// Address of this device's scratch array (the calling thread's current device).
int noalloc_scratch(char **ptr) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, noalloc_scratch_bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error("cudaGetSymbolAddress of the no-alloc scratch failed: %s", cudaGetErrorString(e));
    return PW_ERR_CUDA;
  }
  *ptr = static_cast<char *>(p);
  return PW_OK;
}

}  // namespace pw
