// k_col_f64_v0.cu -- FP64 column kernel of compiled shape 0 (launch.h).
#define COL_REAL double
#define COL_V 0
#include "k_col.inc"
