// elemental_inst_tri3.cu -- the elemental launchers (and with them the kernels) of Tri3.
#include "elemental_kernel.cuh"

HDGX_ELEM_LAUNCHERS(, hdgx::Tri3)
