// Project-written TBB compatibility header: the oneAPI umbrella name.
// Forwards to the shim; <tbb/tbb.h> itself is intentionally absent.
#pragma once
#include "../tbb/nwg_tbb_compat.h"
