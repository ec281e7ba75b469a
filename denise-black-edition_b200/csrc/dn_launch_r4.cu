// Kernel instantiations of FDORDER 8.
#define DN_R 4
#include "dn_launch_impl.cuh"
