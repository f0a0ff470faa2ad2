// stream_reg_dual_kernel instantiations (float64 cells, two Gram entries per lane).
#define DUAL_F64
#define GETTER_NAME get_stream_reg_kernel_f64x2
#include "kernels_stream_reg.inc"
