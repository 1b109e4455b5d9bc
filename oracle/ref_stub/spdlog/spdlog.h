/* Minimal stand-in for the spdlog logging calls made by the reference's codec
 * and IVF headers, so that those headers compile unmodified into oracle/_ref.
 * Logging is discarded. */
#pragma once
namespace spdlog {
template <class... A> inline void info(A &&...) {}
template <class... A> inline void warn(A &&...) {}
template <class... A> inline void error(A &&...) {}
template <class... A> inline void debug(A &&...) {}
}  // namespace spdlog
