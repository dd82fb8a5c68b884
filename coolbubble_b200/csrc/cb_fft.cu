/* cb_fft.cu -- power spectrum (placeholder until the FFT kernels land). */
#include "cb_handle.h"

namespace cb {
struct FftState {};
void free_fft(cb_handle *h) {
    delete h->fft;
    h->fft = nullptr;
}
}  // namespace cb

extern "C" int cb_power_spectrum(cb_handle *h, double *, double *, double *, int) {
    return cb::fail(h, CB_EUNSUPPORTED, "power spectrum not built yet");
}
