// abi_guard.hpp -- keeps C++ exceptions from crossing the C ABI.
//
// Every `extern "C" int` entry point runs its body between NICP_ABI_TRY and
// NICP_ABI_CATCH: a host allocation failure (std::bad_alloc, or a container
// asked for more than it can hold) returns NICP_ENOMEM, any other exception
// NICP_ESTATE.  Nothing is thrown on purpose; the guard only turns what the
// standard library may throw into a status code.
#pragma once

#include <new>
#include <stdexcept>

#include "nicp_gpu.h"

#define NICP_ABI_TRY try {
#define NICP_ABI_CATCH                   \
  }                                      \
  catch (const std::bad_alloc &) {       \
    return NICP_ENOMEM;                  \
  }                                      \
  catch (const std::length_error &) {    \
    return NICP_ENOMEM;                  \
  }                                      \
  catch (...) {                          \
    return NICP_ESTATE;                  \
  }
