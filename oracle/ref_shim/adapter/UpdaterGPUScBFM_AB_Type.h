// ADAPTER SHIM — TEST INFRASTRUCTURE ONLY.
// Stands in for the reference's UpdaterGPUScBFM_AB_Type.h when the reference's own LeMonADE adapter
// (src/pscbfm/GPUScBFM_AB_Type.h, compiled unchanged by oracle/Makefile target `adapter`) is built
// over this engine: the class of that name comes from include/bfm_updater.hpp (the C-ABI). The
// standard headers are the ones the reference's header brought in for the adapter.
#pragma once
#include <ctime>
#include <sstream>

#include "bfm_updater.hpp"
