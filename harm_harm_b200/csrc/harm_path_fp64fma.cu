// harm_path_fp64fma.cu -- the FP64 path's flux and update launchers (harm_path_fp64.cu)
// compiled with FMA contraction and with the inversion's shared reciprocals: every value in
// FP64, as fast as the compiler makes the FP64 code, for comparisons of speed with the mixed
// path (HARM_PREC_FP64_FMA).  Its results differ from the IEEE-ordered FP64 path at round-off
// level.  The kernel instantiations carry their own tag (HARM_TU), so they never share a
// symbol with the other FP64 build.
#define HARM_TU 2
#define HARM_INVERT_FAST_DIV 1
#define HARM_FP64_FMA_TU 1
#include "harm_path_fp64.cu"
