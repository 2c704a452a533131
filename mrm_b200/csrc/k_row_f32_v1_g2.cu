// k_row_f32_v1_g2.cu -- FP32 row kernels of compiled shape 1 (launch.h),
// level 2 (row_kernel's GEN).
#define ROW_REAL float
#define ROW_V 1
#define ROW_GEN 2
#include "k_row.inc"
