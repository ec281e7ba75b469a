// Kernel instantiations of FDORDER 12.
#define DN_R 6
#include "dn_launch_impl.cuh"
