// gcl_guard.h -- keeps C++ exceptions from crossing the C ABI.
//
// The host side of the entry points uses standard containers.  Each entry
// point that does is a function-try-block whose handler returns
// gcl::exception_status(): a failed host allocation becomes GCL_ERR_NOMEM and
// any other exception GCL_ERR_INTERNAL, instead of unwinding into a C,
// ctypes or cgo caller.
#pragma once
#include <new>
#include <stdexcept>

#include "../../include/gcl.h"

namespace gcl {

// Call only from inside a catch handler: classifies the exception in flight.
inline int exception_status() noexcept {
  try {
    throw;
  } catch (const std::bad_alloc&) {
    return GCL_ERR_NOMEM;
  } catch (const std::length_error&) {
    return GCL_ERR_NOMEM;
  } catch (...) {
    return GCL_ERR_INTERNAL;
  }
}

}  // namespace gcl

#define GCL_CATCH_ALL \
  catch (...) {       \
    return gcl::exception_status(); \
  }
