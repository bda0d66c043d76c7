// Extension point of the C++ drop-in (no reference counterpart): chooses the engine
// that bharatopt::GPUFirstOrderSolver runs.  Null restores the default (reference
// engine, or the B2P_ENGINE / B2P_PRECISION / B2P_EPS environment variables).
#pragma once
#include "../../include/b2p.h"

extern "C" void bharatopt_b200_set_engine(const b2p_params* params);
