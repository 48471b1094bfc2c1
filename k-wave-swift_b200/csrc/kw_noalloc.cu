// kw_noalloc.cu — kw_spectral_derivative_noalloc: the spectral derivative of kw_derivative.cpp
// with every device buffer it needs (half-spectrum scratch, FFT twiddle tables, operator vector,
// tile maps, the simulation descriptor) carved out of one file-scope device array instead of
// cudaMalloc. For callers that must not allocate device memory themselves or through the library:
// a host application whose memory manager already owns the device memory, or a loop that cannot
// afford cudaMalloc/cudaFree, whose implicit device-wide synchronisation stalls work on other
// streams.
//
// The array is KW_NOALLOC_SCRATCH_BYTES (16 MiB) of global memory that every GPU which loads this
// library holds until the process exits. All calls share it and it keeps the last call's contents;
// the engine clears every piece it carves before use. Two calls whose work overlaps on the GPU
// (different streams or threads) race on the array.
#include <string>

#include "../../include/kwave_cuda.h"
#include "kw_engine.h"

namespace kw {

static __device__ __align__(256) unsigned char g_noalloc_scratch[KW_NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch on `device`. In host code the array's name is only a host
// stand-in, never a device address; the address comes from cudaGetSymbolAddress with that device
// current. It is looked up on every call rather than cached, so that a device whose context was
// reset (cudaDeviceReset) and re-created gets the address of its new copy of the array.
void* noalloc_scratch(int device) {
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != device) {
        cudaGetLastError();
        throw KwError{KW_ERR_STATE, "scratch set-up needs the context's device current"};
    }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        throw KwError{KW_ERR_CUDA, std::string("cudaGetSymbolAddress of the scratch array failed: ") + cudaGetErrorString(e)};
    }
    return p;
}

}  // namespace kw
