// Force-included (nvcc -include) into every reference source compiled by
// oracle/build.py for the reference CUDA propagator — TEST INFRASTRUCTURE.
//
// The reference selects its precision with `#define SINGLE` in
// src/legacy_compile_options.h:6 (a `#pragma once` header).  Including that
// header first and removing the macro makes every later include of it a no-op,
// so cuda_types.h:13-95 picks cuDoubleComplex / double and the whole
// propagator (cuSPARSE SpMM, cuBLAS axpy/scal, the diagonal-H kernel) runs in
// FP64.  Built with -DHX_REF_KEEP_SINGLE the macro stays and the reference
// runs in its compiled default precision (FP32).  The reference sources
// themselves are compiled unmodified from their own tree; no reference code is
// in this file.
#pragma once
#include "legacy_compile_options.h"
#ifndef HX_REF_KEEP_SINGLE
#undef SINGLE
#endif
