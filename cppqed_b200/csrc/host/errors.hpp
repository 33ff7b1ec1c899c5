// Thread-local last-error message shared by every extern "C" entry point.
#pragma once

#include <exception>
#include <new>
#include <stdexcept>
#include <string>

#include "cqg.h"

namespace cqg {

void setLastError(const std::string& msg);
int fail(int code, const std::string& msg);

// Runs f() and maps C++ exceptions to status codes (the reference throws
// std::runtime_error / std::invalid_argument at the same places).
template <typename F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const std::bad_alloc& e) {
    return fail(CQG_E_NOMEM, std::string("allocation failed: ") + e.what());
  } catch (const std::invalid_argument& e) {
    return fail(CQG_E_INVALID, e.what());
  } catch (const std::exception& e) {
    return fail(CQG_E_INVALID, e.what());
  }
}

}  // namespace cqg
