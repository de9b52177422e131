// btc/btc.h (engine overlay) -- the reference's umbrella header (btc/btc.h:1-45) with its
// operations layer served by libbtc_b200.so.
//
// Put include/btc_overlay ahead of the reference's root on the include path, and include/
// after it:   nvcc -I include/btc_overlay -I include -I <reference root> app.cu -lbtc_b200
// A program written against the reference (its apps/*.cu) then compiles unchanged:
// the reference's common, utils, formats and I/O headers and its CPU triangle count come
// from its own tree, while btc/operations/{convert,bcsr_16x128,bcsr_16x32,btc_core,
// tc_16x128_adaptive,tc_16x32_adaptive}.h resolve to this directory and forward to the
// engine (btc_compat.hpp over the C ABI of btc_c.h).  The list of headers below is the
// reference umbrella's, so the same names are visible.
#pragma once

#include <btc/common/types.h>
#include <btc/common/macros.h>
#include <btc/common/memory.h>
#include <btc/common/constants.h>
#include <btc/common/arithmetic.h>

#include <btc/utils/timer.h>
#include <btc/utils/option.h>
#include <btc/utils/functors.h>
#include <btc/utils/csr_helpers.h>

#include <btc/formats/bitcoo.h>
#include <btc/formats/coo.h>
#include <btc/formats/csr.h>

#include <btc/utils/io/mmio.h>
#include <btc/utils/io/read.h>

#include "operations/convert.h"
#include <btc/operations/triangle_count_cpu.h>
#include "operations/btc_core.h"
