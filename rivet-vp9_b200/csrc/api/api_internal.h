// Shared by the C ABI's translation units.
#pragma once
#include <string>

namespace rv9api {
// Sets the message rv9_last_global_error returns on this thread.
void set_global_error(const std::string& msg);
}  // namespace rv9api
