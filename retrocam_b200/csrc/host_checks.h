// host_checks.h -- argument checks shared by the entry points that take raw
// device pointers: the kernels behind them use 16-, 8- or 4-byte vector
// accesses, and a misaligned address would fault the device, so such calls
// are rejected with RC_ERR_INVALID_ARG instead.
#ifndef RC_HOST_CHECKS_H
#define RC_HOST_CHECKS_H

#include <stddef.h>
#include <stdint.h>

namespace rc {

inline bool aligned_to(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; }

}  // namespace rc

#endif
