// Instantiation unit of the generic derivative kernels: 3-D, VR degree 2, 6 variables.
#include "adjoint_generic.cuh"

DNDSB_GEN_INSTANTIATE_RHS(2, 6)
DNDSB_GEN_INSTANTIATE_VR(2, 6)
