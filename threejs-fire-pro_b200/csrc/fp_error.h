// The calling thread's last error message, which `fp_last_error(NULL)` returns.
#pragma once
#include <string>

// Record `message` for this thread and return `code`.
int fp_set_error(int code, const std::string& message);
