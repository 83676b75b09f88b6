/*
 * XPBD CPU oracle -- TEST INFRASTRUCTURE ONLY (the checker of the CUDA path).
 *
 * A plain-C restatement of the reference solver's per-kernel arithmetic
 * (chunleili/rlmuscleV2, src/muscle/engine.py, constraint/solve_kernels.py,
 * mg/kernel.py, collision/sdf/kernel.py, collision/udcf/kernel.py), built in
 * FP32 (reference precision, reference operation order) and FP64.  Only the
 * test suite, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Parity pinning: the reference cannot execute here (it needs NVIDIA Warp,
 * which is not installed, and its golden frame dumps are Git-LFS pointers), so
 * this oracle is pinned against the known-answer tests the reference's own
 * test files state (tests/test_lion_kernels.py, tests/test_udcf_dcd.py),
 * restated for the current pt3-reference kernels in tests/test_oracle_pins.py.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define REAL float
#define SFX f32
#include "xpbd_oracle_impl.h"
#undef REAL
#undef SFX

#define REAL double
#define SFX f64
#include "xpbd_oracle_impl.h"
#undef REAL
#undef SFX

#include "xpbd_oracle_dcd.h"
#include "xpbd_oracle_bone.h"
