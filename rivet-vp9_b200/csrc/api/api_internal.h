// Shared by the C ABI's translation units.
#pragma once
#include <string>

namespace rv9api {
// Sets the message rv9_last_global_error returns on this thread.
void set_global_error(const std::string& msg);
// Whether this host CPU runs the parser's build (x86-64-v3); sets the global
// error when not. Called before any parser object exists.
bool host_isa_ok();
}  // namespace rv9api
