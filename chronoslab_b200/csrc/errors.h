// Error type and status macros shared by the host C++ and CUDA sources.
#pragma once

#include <stdexcept>
#include <string>

#include "../../include/chronos_b200.h"

namespace chronos {

// Error carried through the C++ layers and turned into a status code at the
// C ABI (no exception crosses it).
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string &msg);

#define CHRONOS_REQUIRE(cond, code, msg)                                            \
  do {                                                                              \
    if (!(cond)) throw ::chronos::Error((code), (msg));                             \
  } while (0)

}  // namespace chronos
