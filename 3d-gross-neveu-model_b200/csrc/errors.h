// errors.h -- the exception that carries a gn_status out of the engine; the
// C-ABI layer turns it into a return code and a thread-local message.
#pragma once
#include <stdexcept>
#include <string>

namespace gn {

struct GnError : std::runtime_error {
  int status;
  GnError(int s, const std::string &m) : std::runtime_error(m), status(s) {}
};

// Records the message gn_last_error() returns (thread-local) and returns status.
int set_last_error(int status, const char *msg);

}  // namespace gn
