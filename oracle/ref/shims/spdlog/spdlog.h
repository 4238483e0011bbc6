// Silent stand-in for the slice of spdlog's API that the reference's logger
// wrapper uses (levels, sinks, a default logger, trace..error).  Building the
// reference's CPU path as a test oracle needs no log output.
#pragma once
#include <memory>
#include <string>
#include <vector>

namespace spdlog {
namespace level {
enum level_enum { trace, debug, info, warn, err, critical, off };
inline level_enum from_str(const std::string&) { return info; }
}  // namespace level

template <typename... Args>
using format_string_t = const char*;

namespace sinks {
class sink {
  public:
    virtual ~sink() = default;
    void set_level(level::level_enum l) { level_ = l; }
    level::level_enum level() const { return level_; }
    void set_pattern(const std::string&) {}
  private:
    level::level_enum level_ = level::info;
};
}  // namespace sinks
using sink_ptr = std::shared_ptr<sinks::sink>;

class logger {
  public:
    logger(std::string, sink_ptr) {}
    template <typename It> logger(std::string, It, It) {}
    void flush_on(level::level_enum) {}
    void flush() {}
    void set_level(level::level_enum) {}
    void set_pattern(const std::string&) {}
};

inline std::shared_ptr<logger>& default_logger_slot() {
    static std::shared_ptr<logger> slot = std::make_shared<logger>("", sink_ptr{});
    return slot;
}
inline void set_default_logger(std::shared_ptr<logger> l) { default_logger_slot() = std::move(l); }
inline std::shared_ptr<logger> default_logger() { return default_logger_slot(); }
inline void set_level(level::level_enum) {}
inline void set_pattern(const std::string&) {}
inline void flush_every(int) {}

template <typename... Args> inline void trace(const char*, Args&&...) {}
template <typename... Args> inline void debug(const char*, Args&&...) {}
template <typename... Args> inline void info(const char*, Args&&...) {}
template <typename... Args> inline void warn(const char*, Args&&...) {}
template <typename... Args> inline void error(const char*, Args&&...) {}
template <typename... Args> inline void critical(const char*, Args&&...) {}
}  // namespace spdlog
