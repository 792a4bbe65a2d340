// Error type of the host library.  Mirrors nec_exception
// (src/nec_exception.h:27-63): the C API catches it, stores the message in a
// process-global string and returns 1 (src/libNEC.cpp:27-30).
#pragma once
#include <sstream>
#include <stdexcept>
#include <string>

namespace necb {

struct nec_error : std::runtime_error {
  explicit nec_error(const std::string& m) : std::runtime_error(m) {}
};

template <typename... Args>
[[noreturn]] inline void fail(Args&&... parts) {
  std::ostringstream os;
  (os << ... << parts);
  throw nec_error(os.str());
}

}  // namespace necb
