// Kernel instantiations of FDORDER 6.
#define DN_R 3
#include "dn_launch_impl.cuh"
