// Shared host-side helpers: thread-local error message and status plumbing.
#pragma once
#include <string>

namespace rmt3d {
int fail(int code, const std::string &msg);
}
