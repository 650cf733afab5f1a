// C ABI: ray tracing, Jacobian, CGLS and model update (include/tomo_b200.h).
#include "context.hpp"

extern "C" {

// Releases the tomography-side device buffers of a context (called by tomo_ctx_destroy).
void tomo_release_tomography(tomo_ctx *ctx) { (void)ctx; }

}  // extern "C"
