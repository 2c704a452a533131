// k_row_f32_v3_g2.cu -- FP32 row kernels of compiled shape 3 (launch.h),
// level 2 (row_kernel's GEN).
#define ROW_REAL float
#define ROW_V 3
#define ROW_GEN 2
#include "k_row.inc"
