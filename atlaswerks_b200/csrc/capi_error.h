// capi_error.h — the thread-local message behind aw_last_error().
#pragma once

#include <string>

namespace aw {
void set_last_error(const std::string &msg);
}
