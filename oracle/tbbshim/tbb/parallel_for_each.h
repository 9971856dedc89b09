// TBB-API shim header (oracle test infrastructure); everything lives in _shim_core.h.
#pragma once
#include "tbb/_shim_core.h"
