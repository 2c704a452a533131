// k_creg_v2.cu -- register column kernel of compiled shape 2 (launch.h kCreg).
#define CREG_V 2
#include "k_creg.inc"
