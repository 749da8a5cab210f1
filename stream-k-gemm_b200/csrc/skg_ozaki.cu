// Ozaki split-precision path.
#include "skg_ozaki.h"

namespace skg {

int ozaki_gemm_packed(int64_t, int64_t, int64_t, const double*, const double*, double*, int64_t,
                      double, double, skgemm_options_t*, cudaStream_t) {
  return fail(SKGEMM_ERR_UNSUPPORTED, "Ozaki path not built yet");
}
int ozaki_syrk_packed(int64_t, int64_t, const double*, double*, int64_t, double, double,
                      skgemm_options_t*, cudaStream_t) {
  return fail(SKGEMM_ERR_UNSUPPORTED, "Ozaki path not built yet");
}
int ozaki_rot(int64_t, int64_t, const double*, const double*, double*, skgemm_options_t*,
              cudaStream_t) {
  return fail(SKGEMM_ERR_UNSUPPORTED, "Ozaki path not built yet");
}
int ozaki_consume_error(DeviceState*, cudaStream_t) { return SKGEMM_OK; }

}  // namespace skg
