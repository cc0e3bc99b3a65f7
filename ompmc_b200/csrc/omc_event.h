// Event-based FP32 transport form (omc_event.cu).
#pragma once
#include "omc_engine.h"

namespace omc {
int event_run_beam(omc_engine *e, const omc_beam *b, long nper, int nbatch, uint64_t seed, double *sum, double *sum2,
                   double *src_energy, KernelStats &ks);
void event_release(omc_engine *e);
template <typename R>
BeamSrc<R> beam_setup(const omc_engine *e, const omc_beam *b);
int fold(omc_engine *e, double *work, double *sum, double *sum2, long n, double scale);
}  // namespace omc
