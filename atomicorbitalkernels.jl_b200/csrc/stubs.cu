// stubs.cu -- entry points not yet implemented in this build: they report
// AOK_ERR_UNSUPPORTED instead of computing anything.
#include "aok_internal.h"
using namespace aok;
extern "C" {
int aok_overlap3c_gb(aok_plan*, void*, const int64_t*, const int64_t*, const void*, const void*, const void*,
                     const void*, const void*, int64_t, void*) {
    return set_error(AOK_ERR_UNSUPPORTED, "aok_overlap3c_gb: not implemented yet");
}
}
