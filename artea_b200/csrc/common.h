// Shared host helpers of the C-ABI: thread-local error text and status codes.
#pragma once

#include <string>

#include "../../include/artea_gpu.h"

namespace artea_gpu {

// Records msg as the calling thread's last error and returns code.
int fail(int code, const std::string& msg);

}  // namespace artea_gpu
