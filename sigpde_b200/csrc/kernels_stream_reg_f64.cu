// stream_reg_kernel instantiations with float64 cells.
#define CELL_T double
#define GETTER_NAME get_stream_reg_kernel_f64
#include "kernels_stream_reg.inc"
