// k_row_f32_v4.cu -- FP32 row kernels of compiled shape 4 (launch.h).
#define ROW_REAL float
#define ROW_V 4
#include "k_row.inc"
