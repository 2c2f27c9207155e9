// defs.hh parses vectors from the command line and throws the parser's
// exception on bad input; the shape functions use neither.
#pragma once
#include <stdexcept>
#include <string>
namespace TCLAP {
struct ArgParseException : std::runtime_error {
  explicit ArgParseException(const std::string &s) : std::runtime_error(s) {}
};
}
