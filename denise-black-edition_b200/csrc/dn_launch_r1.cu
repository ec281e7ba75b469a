// Kernel instantiations of FDORDER 2.
#define DN_R 1
#include "dn_launch_impl.cuh"
