// Fused Landau step kernels for 96^3 grids in float (all variant counts and schedules).
#include "landau_fused_kernels.cuh"
MEU_LF_INSTANTIATE(float, 96)
