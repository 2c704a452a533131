// k_row_f32_v0.cu -- FP32 row kernels of compiled shape 0 (launch.h).
#define ROW_REAL float
#define ROW_V 0
#include "k_row.inc"
