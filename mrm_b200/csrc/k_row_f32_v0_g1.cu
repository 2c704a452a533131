// k_row_f32_v0_g1.cu -- FP32 row kernels of compiled shape 0 (launch.h),
// level 1 (row_kernel's GEN).
#define ROW_REAL float
#define ROW_V 0
#define ROW_GEN 1
#include "k_row.inc"
