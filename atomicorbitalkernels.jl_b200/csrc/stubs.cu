// stubs.cu -- entry points not yet implemented in this build: they report
// AOK_ERR_UNSUPPORTED instead of computing anything.
#include "aok_internal.h"
using namespace aok;
extern "C" {
int aok_overlap3c_gb(aok_plan*, void*, const int64_t*, const int64_t*, const void*, const void*, const void*,
                     const void*, const void*, int64_t, void*) {
    return set_error(AOK_ERR_UNSUPPORTED, "aok_overlap3c_gb: not implemented yet");
}
int aok_orbitals_create(aok_orbitals**, int64_t, int64_t, int64_t, const int64_t*, int64_t, const int64_t*,
                        const int64_t*, int64_t, int, int) {
    return set_error(AOK_ERR_UNSUPPORTED, "aok_orbitals_create: not implemented yet");
}
int aok_orbitals_destroy(aok_orbitals*) { return AOK_OK; }
int aok_evaluate(aok_orbitals*, void*, const void*, const int64_t*, const void*, const void*, int64_t, double,
                 void*) {
    return set_error(AOK_ERR_UNSUPPORTED, "aok_evaluate: not implemented yet");
}
int aok_evaluate_ed(aok_orbitals*, void*, void*, const void*, const int64_t*, const void*, const void*, int64_t,
                    double, void*) {
    return set_error(AOK_ERR_UNSUPPORTED, "aok_evaluate_ed: not implemented yet");
}
int aok_evaluate_pullback(aok_orbitals*, void*, void*, void*, const void*, const void*, const int64_t*,
                          const void*, const void*, int64_t, double, void*) {
    return set_error(AOK_ERR_UNSUPPORTED, "aok_evaluate_pullback: not implemented yet");
}
}
