// prefilter_fwd.cu — the prefiltered forward kernels (k_forward_prefilter and its batched
// form), compiled from prefilter.cu in a translation unit of their own so that their
// root solves can differ from the rest of the library: here the crate's formulas
// (DVG_EXACT_ROOT_SOLVES), without the certified f32 + Newton shortcuts of
// winding_newton.cuh.  At this kernel's 64-register budget the shortcuts cost more than
// they save (mixed 512x512 scene, 4x4 spp: 43.5 ms with them, 39.6 without), while the
// prefiltered interior, with 168 registers, runs faster with the winding one (66.9
// against 71.8 ms).
#define DVG_EXACT_ROOT_SOLVES 1
#define DVG_PREFILTER_FORWARD 1
#include "prefilter.cu"
