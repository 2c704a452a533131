// k_col_f32_v0.cu -- FP32 column kernel of compiled shape 0 (launch.h).
#define COL_REAL float
#define COL_V 0
#include "k_col.inc"
