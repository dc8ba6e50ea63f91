/* ams_hserscspgemm: C = A·B with the hsersc accumulator on one GPU; the process
 * interface and log text of the reference's src/ams_hserscspgemm.c (see cas_driver.h). */
#include "cas_driver.h"

int main(int argc, char **argv) { return cas_driver_main(argc, argv, CAS_ACC_HSERSC, "ams_hserscspgemm"); }
