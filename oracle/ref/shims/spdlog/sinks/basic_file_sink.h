// Silent stand-in for spdlog's file sink (see ../spdlog.h).
#pragma once
#include <string>
#include "../spdlog.h"
namespace spdlog { namespace sinks {
class basic_file_sink_mt : public sink {
  public:
    basic_file_sink_mt(const std::string&, bool = false) {}
};
}}  // namespace spdlog::sinks
