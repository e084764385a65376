// cmd_internal.h -- shared helpers of the C-ABI implementation (not installed).
#pragma once

#include <string>

namespace cmd {

// Records `msg` as this host thread's last error and returns `code`.
int fail(int code, const std::string& msg);
// Clears the last error (called at the start of every public entry point).
void clear_error();

}  // namespace cmd
