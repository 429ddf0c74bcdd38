// Entry points of the C ABI whose subsystems are not built yet.  Each
// returns DL_ERR_UNSUPPORTED with a message naming what is missing.
#include <string>

#include "../../include/dynlattice.h"

namespace dl {
extern thread_local std::string g_last_error;
}

namespace {
int unsupported(const char *what) {
  dl::g_last_error = std::string(what) + " is not available in this build";
  return DL_ERR_UNSUPPORTED;
}
}  // namespace

DL_API int dl_create_from_pro(const char *, int, dl_handle **) { return unsupported(".pro input"); }
