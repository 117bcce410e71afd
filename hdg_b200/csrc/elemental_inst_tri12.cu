// elemental_inst_tri12.cu -- the elemental launchers (and with them the kernels) of Tri1, Tri2, Tet1.
#include "elemental_kernel.cuh"

HDGX_ELEM_LAUNCHERS(, hdgx::Tri1)
HDGX_ELEM_LAUNCHERS(, hdgx::Tri2)
HDGX_ELEM_LAUNCHERS(, hdgx::Tet1)
