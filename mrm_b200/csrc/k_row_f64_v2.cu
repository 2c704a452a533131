// k_row_f64_v2.cu -- FP64 row kernels of compiled shape 2 (launch.h).
#define ROW_REAL double
#define ROW_V 2
#include "k_row.inc"
