// The error-message hook of the CPU scene generator (antiradiancecuts_b200/csrc/scene_gen.cpp) for
// its stand-alone build, oracle/libinputs.so: the benchmark's CPU arm makes its synthetic inputs
// with the same generator source without loading the GPU library.  Test infrastructure only.
#include <string>

namespace {
thread_local std::string g_message;
}

namespace arc {
void set_last_error(const std::string& msg) { g_message = msg; }
}  // namespace arc

extern "C" const char* arc_last_error(void) { return g_message.c_str(); }
