// Kernel instantiations of FDORDER 4.
#define DN_R 2
#include "dn_launch_impl.cuh"
