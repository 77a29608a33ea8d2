// Test infrastructure for the oracle build only.  The reference's Logger.hpp routes its
// ZS_* log macros to plog, which lives in the absent zpc_tpls submodule.  Logging is not on
// the MPM arithmetic path, so the oracle build maps the same macro names to stderr prints.
#pragma once
#include <cstdio>

#define ZS_LOG_SHIM_PRINT(tag, ...) std::fprintf(stderr, "[zpc %s] %s:%d\n", tag, __FILE__, __LINE__)
#define ZS_FATAL(...) ZS_LOG_SHIM_PRINT("fatal", __VA_ARGS__)
#define ZS_INFO(...) ZS_LOG_SHIM_PRINT("info", __VA_ARGS__)
#define ZS_WARN(...) ZS_LOG_SHIM_PRINT("warn", __VA_ARGS__)
#define ZS_ERROR(...) ZS_LOG_SHIM_PRINT("error", __VA_ARGS__)
#define ZS_ERROR_IF(condition, ...) \
  if (condition) {                  \
    ZS_ERROR(__VA_ARGS__);          \
  }
#define ZS_WARN_IF(condition, ...) \
  if (condition) {                 \
    ZS_WARN(__VA_ARGS__);          \
  }
