// elemental_inst_tet2.cu -- the elemental launchers (and with them the kernels) of Tet2.
#include "elemental_kernel.cuh"

HDGX_ELEM_LAUNCHERS(, hdgx::Tet2)
