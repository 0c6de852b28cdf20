/* TEST INFRASTRUCTURE ONLY (oracle): storage for the shim's per-thread NDRange index. */
#include "clshim.h"
namespace clshim {
thread_local size_t gid[3];
}
