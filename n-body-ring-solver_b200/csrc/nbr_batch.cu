// nbr_batch.cu -- batched independent systems (nbr_batch_*).
#include "nbr.h"
#include "nbr_ctx.h"

using namespace nbr;

void nbr::BatchState::release() {
  s.release();
  dfree(d_poff);
  dfree(d_nreal);
  dfree(d_sys_of_tile);
  dfree(d_items);
  dfree(d_head);
  dfree(d_red);
  *this = BatchState();
}

extern "C" {
int nbr_batch_upload(nbr_ctx* c, size_t, const size_t*, const double*, const double*,
                     const double*, const double*, const double*, const double*, const double*) {
  return fail(c, NBR_ERR_UNSUPPORTED, "batched systems not built yet");
}
int nbr_batch_download(nbr_ctx* c, double*, double*, double*, double*, double*, double*) {
  return fail(c, NBR_ERR_UNSUPPORTED, "batched systems not built yet");
}
int nbr_batch_forces(nbr_ctx* c, int, double, double, int, double*, double*, double*) {
  return fail(c, NBR_ERR_UNSUPPORTED, "batched systems not built yet");
}
int nbr_batch_run(nbr_ctx* c, int, double, size_t, double, double, nbr_run_stats*) {
  return fail(c, NBR_ERR_UNSUPPORTED, "batched systems not built yet");
}
int nbr_batch_diagnostics(nbr_ctx* c, double, double, nbr_diag*) {
  return fail(c, NBR_ERR_UNSUPPORTED, "batched systems not built yet");
}
}
