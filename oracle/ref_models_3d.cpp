// SymPhas's models on 3D stencils: the configurations' Stencil3d2h<7,10,25>
// and SymPhas's default Stencil3d2h<> = <15,10,25>
#include "symphas_ref.h"
SYMREF_REGISTER(m3a, 3, 2, Stencil3d2h, 7, 10, 25, 1, 1)
SYMREF_REGISTER(m3b, 3, 2, Stencil3d2h, 15, 10, 25, 1, 1)
