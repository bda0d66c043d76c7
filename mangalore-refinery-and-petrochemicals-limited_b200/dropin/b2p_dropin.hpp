// Extension point of the C++ drop-in (no reference counterpart): chooses the engine
// that bharatopt::GPUFirstOrderSolver runs.  Null restores the default (reference
// engine, or the B2P_ENGINE / B2P_PRECISION / B2P_EPS environment variables).
#pragma once
#include "../../include/b2p.h"

extern "C" void bharatopt_b200_set_engine(const b2p_params* params);

// Extension point (no reference counterpart): 1 selects the direct setup of
// bharatopt::GPUFirstOrderSolver (one threaded pass from the model's rows to the
// standard form, no validator / presolve, the Halpern engine), 0 the reference's front
// end, -1 the B2P_SETUP environment variable (B2P_SETUP=direct).
extern "C" void bharatopt_b200_set_setup(int direct);
