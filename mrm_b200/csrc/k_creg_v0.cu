// k_creg_v0.cu -- register column kernel of compiled shape 0 (launch.h kCreg).
#define CREG_V 0
#include "k_creg.inc"
