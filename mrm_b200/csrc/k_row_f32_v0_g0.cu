// k_row_f32_v0_g0.cu -- FP32 row kernels of compiled shape 0 (launch.h),
// level 0 (row_kernel's GEN).
#define ROW_REAL float
#define ROW_V 0
#define ROW_GEN 0
#include "k_row.inc"
