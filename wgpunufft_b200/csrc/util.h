// Thread-local error messages and launch accounting.
#pragma once

#include <cstdint>
#include <string>

namespace b200nufft {

void set_last_error(const std::string& message);
const char* last_error();
uint64_t launch_count();

}  // namespace b200nufft
