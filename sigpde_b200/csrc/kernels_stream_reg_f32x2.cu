// stream_reg_paired_kernel instantiations (float32 cells, two pairs per lane).
#define PAIRED_F32
#define GETTER_NAME get_stream_reg_kernel_f32x2
#include "kernels_stream_reg.inc"
