// Silent stand-in for spdlog's colour console sink (see ../spdlog.h).
#pragma once
#include "../spdlog.h"
namespace spdlog { namespace sinks {
class stdout_color_sink_mt : public sink {};
class stderr_color_sink_mt : public sink {};
}}  // namespace spdlog::sinks
