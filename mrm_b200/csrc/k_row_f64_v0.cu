// k_row_f64_v0.cu -- FP64 row kernels of compiled shape 0 (launch.h).
#define ROW_REAL double
#define ROW_V 0
#include "k_row.inc"
