// Event-based FP32 transport form.
#include "omc_event.h"

namespace omc {
int event_run_beam(omc_engine *e, const omc_beam *, long, int, uint64_t, double *, double *, double *, KernelStats &) {
    return set_err(e, OMC_E_RANGE, "event form not built yet");
}
void event_release(omc_engine *) {}
}  // namespace omc
