// Exception-to-status translation for the C ABI entry points.
#pragma once
#include <new>
#include <string>

#include "../../include/sipg_b200.h"
#include "runtime.hpp"

namespace sipg {
void set_last_error(const std::string& s);

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return SIPG_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.status;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return SIPG_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return SIPG_INVALID_ARG;
  }
}
}  // namespace sipg
