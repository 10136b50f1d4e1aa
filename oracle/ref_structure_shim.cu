// ref_structure_shim.cu -- TEST INFRASTRUCTURE ONLY (built by oracle/ref.mk).
//
// Compiles the reference's structure.cu where it lies, with one change of
// behaviour: its `cuchk` (cuda_helpers.h:18-21) exits the process on a CUDA
// error, and encodingMeta::init (structure.cu:113-135) copies the block count
// to constant memory through it.  The host checker runs where no GPU may be
// present, so here a failed copy is ignored; nothing the plan pins depends on
// that copy.
#include "cuda_helpers.h"
#undef cuchk
#define cuchk(ans) ((void)(ans))
#include "structure.cu"
