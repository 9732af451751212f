// errors.hpp -- status/message plumbing shared by the C ABI translation units.
#pragma once

#include <string>

namespace mlem {

// The message of the last failed call on this thread (mlem_global_error()).
std::string& global_error();

// printf-style: store the message in *slot (may be null) and in the
// thread's global error; return `status`.
int set_error(std::string* slot, int status, const char* fmt, ...)
    __attribute__((format(printf, 3, 4)));

}  // namespace mlem
