// batch.cu -- cyc_batch_fit (filled in by the batched persistent solver)
#include "internal.cuh"

extern "C" int cyc_batch_fit(cyc_dataset* ds, const cyc_prior* prior, const cyc_fit_spec* specs, int F,
                             const cyc_control* control, cyc_fit_result* out) {
    (void)ds; (void)prior; (void)specs; (void)F; (void)control; (void)out;
    cyc::set_error("cyc_batch_fit: not built yet");
    return CYC_ERR_UNSUPPORTED;
}
