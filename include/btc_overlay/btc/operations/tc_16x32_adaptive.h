// btc/operations/tc_16x32_adaptive.h (engine overlay): the Bit-BSR structs, convert_coo_to_bcsr_* and
// count_triangles_*_adaptive of the reference, served by libbtc_b200.so (see btc/btc.h).
#pragma once

#include "btc_compat.hpp"
