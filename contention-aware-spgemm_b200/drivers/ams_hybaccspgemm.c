/* ams_hybaccspgemm: C = A·B with the hybacc accumulator on one GPU; the process
 * interface and log text of the reference's src/ams_hybaccspgemm.c (see cas_driver.h). */
#include "cas_driver.h"

int main(int argc, char **argv) { return cas_driver_main(argc, argv, CAS_ACC_HYBACC, "ams_hybaccspgemm"); }
