// Kernel instantiations of FDORDER 10.
#define DN_R 5
#include "dn_launch_impl.cuh"
