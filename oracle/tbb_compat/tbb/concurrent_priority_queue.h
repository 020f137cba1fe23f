// Project-written TBB compatibility header: forwards to nwg_tbb_compat.h.
#pragma once
#include "nwg_tbb_compat.h"
