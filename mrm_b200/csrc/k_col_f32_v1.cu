// k_col_f32_v1.cu -- FP32 column kernel of compiled shape 1 (launch.h).
#define COL_REAL float
#define COL_V 1
#include "k_col.inc"
