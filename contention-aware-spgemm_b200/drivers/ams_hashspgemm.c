/* ams_hashspgemm: C = A·B with the hash accumulator on one GPU; the process
 * interface and log text of the reference's src/ams_hashspgemm.c (see cas_driver.h). */
#include "cas_driver.h"

int main(int argc, char **argv) { return cas_driver_main(argc, argv, CAS_ACC_HASH, "ams_hashspgemm"); }
