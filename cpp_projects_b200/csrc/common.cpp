// Error reporting shared by every entry point.
#include <cstdio>

#include "internal.h"

namespace bfs {
namespace {
thread_local char g_last_error[1024] = "";
}

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

bfs_status fail(bfs_status st, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return st;
}

const char* last_error() { return g_last_error; }

}  // namespace bfs

extern "C" const char* bfs_last_error(void) { return bfs::last_error(); }
extern "C" const char* bfs_version(void) { return "bfs-b200 0.1 (sm_100a)"; }
