// Persistent ensemble kernel in double (every grid size of the fused path, one order parameter).
#include "ens_persist_impl.cuh"
MEU_PK_INSTANTIATE(double)
