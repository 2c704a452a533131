// k_row_f32_v2.cu -- FP32 row kernels of compiled shape 2 (launch.h).
#define ROW_REAL float
#define ROW_V 2
#include "k_row.inc"
