// TBB-API shim umbrella header (oracle test infrastructure).
#pragma once
#include "tbb/_shim_core.h"
