// Internal helpers shared by the translation units of the library.
#pragma once
#include <string>

// Record `msg` as the calling thread's last error and return `code`.
int pbpic_internal_fail(int code, const std::string& msg);
// Count one kernel launch (reported by pbpic_kernel_launches).
void pbpic_internal_count_launch();
