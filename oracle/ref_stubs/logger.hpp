// Stand-in for the reference's quill logger (include/logger.hpp), used only to
// compile the reference's own kernels as the parity pin. Logging is dropped.
#pragma once
#include <string>
namespace quill { class Logger; }
namespace YallaSQL {
inline quill::Logger* getLogger(const std::string&) { return nullptr; }
}  // namespace YallaSQL
#define LOG_ERROR(...) ((void)0)
#define LOG_WARNING(...) ((void)0)
#define LOG_INFO(...) ((void)0)
#define LOG_DEBUG(...) ((void)0)
#define LOG_TRACE_L1(...) ((void)0)
#define LOG_TRACE_L2(...) ((void)0)
#define LOG_TRACE_L3(...) ((void)0)
