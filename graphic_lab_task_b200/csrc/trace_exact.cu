// trace_exact.cu — the bit-exact build of the trace kernels.  Compiled with
// -fmad=false (plus IEEE division and square root), so every float operation
// rounds exactly like the reference CPU path built with -ffp-contract=off.
#include <algorithm>
#define LRT_NS lrt_exact
#include "trace_impl.cuh"
