// Drop-in glue: MPLB's StreamCollision / UpdateMacroVars(3D) /
// CalcResidualError on the B200 path.  Compiled into the reference's own
// build (with its headers and OPS) with -DMPLB_B200, together with three
// early returns in the reference that route its functions here:
// StreamCollision (Src/evolution.cpp) calls mplbgpu_dropin::StreamCollision,
// and UpdateMacroVars(3D) (Src/model_wrapper.cpp) and CalcResidualError
// (Src/flowfield_wrapper.cpp) call the glue's versions when Active().
//
// On the first StreamCollision the glue reads what the setup API holds
// (g_Block() and each Block::Neighbors(), BlockBoundaries(), g_Components(),
// TimeStep(), SoundSpeed(), g_MacroBodyforce(), g_MacroVars(), g_f()),
// creates an mplbgpu context and sets its state - from the initial
// macroscopic fields when the first step is at time 0 (f = feq of them, and
// they are the residual's previous values as in the reference), else by
// uploading f (restart); from then on the distributions stay on the GPU and
// StreamCollision only queues the step's kernels (no host wait).
// UpdateMacroVars copies the moments (and, unless MPLB_B200_SYNC_F=0,
// the distributions) back into the reference's dats so that Iterate's HDF5
// writers see current data.  MPLB_B200_PRECISION=fp32|fp16 selects a
// shifted storage form (default fp64, bit-identical to the reference).
#ifndef MPLBGPU_DROPIN_H
#define MPLBGPU_DROPIN_H

#include "type.h"

namespace mplbgpu_dropin {

// True once the GPU context exists (after the first StreamCollision).
bool Active();

// Replaces the body of StreamCollision(time) (Src/evolution.cpp:137-193).
void StreamCollision(const Real time);

// Replaces the body of SwapStreamCollision(time) (Src/evolution.cpp:
// 195-252); the context was created with the swap scheme (Scheme()).
void SwapStreamCollision(const Real time);

// Replaces UpdateMacroVars3D / UpdateMacroVars when Active().
void UpdateMacroVars();

// Replaces CalcResidualError (Src/flowfield_wrapper.cpp:31-89) when Active().
void CalcResidualError();

// Waits until the GPU has done every step queued so far (StreamCollision
// returns as soon as its kernels are queued).
void Synchronize();

// Frees the GPU context.
void Release();

}  // namespace mplbgpu_dropin

#endif
