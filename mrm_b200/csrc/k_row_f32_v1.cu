// k_row_f32_v1.cu -- FP32 row kernels of compiled shape 1 (launch.h).
#define ROW_REAL float
#define ROW_V 1
#include "k_row.inc"
