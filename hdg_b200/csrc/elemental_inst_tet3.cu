// elemental_inst_tet3.cu -- the elemental launchers (and with them the kernels) of Tet3.
#include "elemental_kernel.cuh"

HDGX_ELEM_LAUNCHERS_FP64(, hdgx::Tet3)
