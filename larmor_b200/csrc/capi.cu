// Library-wide C-ABI entry points: error reporting and version.
#include <string>

#include "common.cuh"

namespace lar {

namespace {
thread_local std::string last_error;
}

void set_error(const std::string& message) { last_error = message; }

}  // namespace lar

extern "C" {

const char* lar_last_error(void) { return lar::last_error.c_str(); }

const char* lar_version(void) { return "larmor_b200 0.1.0 (sm_100a)"; }

}  // extern "C"
