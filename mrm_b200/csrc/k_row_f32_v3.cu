// k_row_f32_v3.cu -- FP32 row kernels of compiled shape 3 (launch.h).
#define ROW_REAL float
#define ROW_V 3
#include "k_row.inc"
