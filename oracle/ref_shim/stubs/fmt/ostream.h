// Minimal stand-in for the fmt library so that the reference's leaf headers
// (common.h) compile without the real dependency. Only the names the
// reference's hot-path headers reference are provided; formatting is a no-op.
#pragma once
#include <string>
#include <ostream>
namespace fmt {
template <class... A> inline std::string format(A&&...) { return std::string(); }
}
