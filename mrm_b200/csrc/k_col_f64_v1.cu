// k_col_f64_v1.cu -- FP64 column kernel of compiled shape 1 (launch.h).
#define COL_REAL double
#define COL_V 1
#include "k_col.inc"
