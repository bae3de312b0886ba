// SymPhas's models on 2D stencils: the configurations' Stencil2d2h<5,6,13>,
// SymPhas's default Stencil2d2h<> = <9,6,13>, and Stencil2d4h<9,14,21>
#include "symphas_ref.h"
SYMREF_REGISTER(m2a, 2, 2, Stencil2d2h, 5, 6, 13, 1, 1)
SYMREF_REGISTER(m2b, 2, 2, Stencil2d2h, 9, 6, 13, 1, 1)
SYMREF_REGISTER(m2c, 2, 4, Stencil2d4h, 9, 14, 21, 1, 1)
