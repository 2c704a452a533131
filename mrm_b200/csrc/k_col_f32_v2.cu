// k_col_f32_v2.cu -- FP32 column kernel of compiled shape 2 (launch.h).
#define COL_REAL float
#define COL_V 2
#include "k_col.inc"
