// elemental_inst_tri4.cu -- the elemental launchers (and with them the kernels) of Tri4.
#include "elemental_kernel.cuh"

HDGX_ELEM_LAUNCHERS(, hdgx::Tri4)
