// stream_reg_kernel instantiations with float32 cells.
#define CELL_T float
#define GETTER_NAME get_stream_reg_kernel_f32
#include "kernels_stream_reg.inc"
