// Fused Landau step kernels for 48^3 grids in double (all variant counts and schedules).
#include "landau_fused_kernels.cuh"
MEU_LF_INSTANTIATE(double, 48)
