// Shared host helpers: thread-local error message and status plumbing.
#pragma once
#include <cstdarg>
#include <cstdio>
#include <string>

namespace gm {

std::string &last_error();

// Records a formatted message for gm_last_error() and returns `code`.
int fail(int code, const char *fmt, ...);

}  // namespace gm
