// Thread-local error text behind og_last_error().
#pragma once
#include <string>

#include "../../../include/origami_gpu.h"

// Records `msg` as this thread's last error and returns `st`.
og_status og_fail(og_status st, const std::string& msg);
