// Shared host-side helpers: status codes, the thread-local error string and a
// guard that turns C++ exceptions into status codes so that nothing throws
// across the C ABI.
#pragma once

#include <cstdint>
#include <exception>
#include <new>
#include <string>

#include "../../include/beep3_b200.h"

#define BP_API __attribute__((visibility("default")))

namespace bp {

void set_error(const std::string& msg);

inline int32_t fail(int32_t code, const std::string& msg) {
  set_error(msg);
  return code;
}

template <typename F>
int32_t guarded(F&& f) {
  try {
    return f();
  } catch (const std::bad_alloc&) {
    return fail(BP_ERR_NOMEM, "host allocation failed");
  } catch (const std::invalid_argument& e) {
    return fail(BP_ERR_INVALID, e.what());
  } catch (const std::exception& e) {
    return fail(BP_ERR_INTERNAL, e.what());
  } catch (...) {
    return fail(BP_ERR_INTERNAL, "unknown exception");
  }
}

}  // namespace bp
