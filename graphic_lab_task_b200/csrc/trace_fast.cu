// trace_fast.cu — the FMA-contracted build of the trace kernels (-fmad=true).
// Same code as trace_exact.cu; results agree with the reference to the
// tolerances of the hot-path specification (t 1e-5 relative, normals 1e-4).
#include <algorithm>
#define LRT_NS lrt_fast
#include "trace_impl.cuh"
