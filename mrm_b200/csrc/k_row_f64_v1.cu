// k_row_f64_v1.cu -- FP64 row kernels of compiled shape 1 (launch.h).
#define ROW_REAL double
#define ROW_V 1
#include "k_row.inc"
