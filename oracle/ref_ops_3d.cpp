// operator checks on every 3D point set of SymPhas's 2nd-order stencils (one
// set varied, the others at the configurations' defaults)
#include "symphas_ref.h"
SYMREF_REGISTER(o3a, 3, 2, Stencil3d2h, 19, 10, 25, 0, 1)
SYMREF_REGISTER(o3b, 3, 2, Stencil3d2h, 21, 10, 25, 0, 1)
SYMREF_REGISTER(o3c, 3, 2, Stencil3d2h, 27, 10, 25, 0, 1)
SYMREF_REGISTER(o3d, 3, 2, Stencil3d2h, 7, 12, 25, 0, 1)
SYMREF_REGISTER(o3e, 3, 2, Stencil3d2h, 7, 28, 25, 0, 1)
SYMREF_REGISTER(o3f, 3, 2, Stencil3d2h, 7, 36, 25, 0, 1)
SYMREF_REGISTER(o3g, 3, 2, Stencil3d2h, 7, 40, 25, 0, 1)
SYMREF_REGISTER(o3h, 3, 2, Stencil3d2h, 7, 10, 21, 0, 1)
SYMREF_REGISTER(o3i, 3, 2, Stencil3d2h, 7, 10, 41, 0, 1)
SYMREF_REGISTER(o3j, 3, 2, Stencil3d2h, 7, 10, 52, 0, 1)
SYMREF_REGISTER(o3k, 3, 2, Stencil3d2h, 7, 10, 57, 0, 1)
