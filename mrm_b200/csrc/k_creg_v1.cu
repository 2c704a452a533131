// k_creg_v1.cu -- register column kernel of compiled shape 1 (launch.h kCreg).
#define CREG_V 1
#include "k_creg.inc"
