/* Swift system-library shim for libkwave_cuda.so (the B200 k-space solver's C ABI).
 *
 * A k-wave-swift checkout adds this directory as Sources/CKWaveCUDA next to Sources/CHDF5, with
 * include/kwave_cuda.h of this repository on the include path (or copied next to this file), and
 * the directory holding libkwave_cuda.so on the linker path (swift build -Xlinker -L<dir>). */
#ifndef CKWAVECUDA_SHIM_H
#define CKWAVECUDA_SHIM_H
#include "kwave_cuda.h"
#endif
