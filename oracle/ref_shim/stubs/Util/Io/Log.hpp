// Minimal logging stand-in for the reference's spdlog wrapper (Util/Io/Log.hpp).
// The oracle build only needs the names; every call is a no-op.
#pragma once
#include <string>
namespace medyan { namespace log {
template <class... A> inline void debug(A&&...) {}
template <class... A> inline void info(A&&...) {}
template <class... A> inline void warn(A&&...) {}
template <class... A> inline void error(A&&...) {}
template <class... A> inline void critical(A&&...) {}
}}
