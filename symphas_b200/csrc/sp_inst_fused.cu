/*
 * sp_inst_fused.cu -- kernels of the FUSED form (bilap = lap o lap, merged
 * derivatives, staged operands); FMA contraction allowed.  For point sets
 * where bilap is not lap o lap, the FUSED key runs the exact term order
 * compiled with FMA; so does every Stencil2d4h key (no 4th-order bilaplacian
 * is a Laplacian applied twice).
 */
#include "sp_launch.cuh"

#define SP_FUSED_SET(T, DT)                                                \
  SP_REG2(SPK_A, SPK_FUSED, MF_A_fused, T, DT, 5, 6, 13);                            \
  SP_REG2(SPK_B, SPK_FUSED, MF_B_fused, T, DT, 5, 6, 13);                            \
  SP_REG2(SPK_C, SPK_FUSED, MF_C_fused, T, DT, 5, 6, 13);                            \
  SP_REG2(SPK_AMK, SPK_FUSED, MF_AMK_fused, T, DT, 5, 6, 13);                        \
  SP_REG2(SPK_BMK, SPK_FUSED, MF_BMK_fused, T, DT, 5, 6, 13);                        \
  SP_REG2X(SPK_ENS_AB, SPK_FUSED, MF_AMK_fused, MF_BMK_fused, T, DT, 5, 6, 13);      \
  SP_REG3(SPK_A, SPK_FUSED, MF_A_fused, T, DT, 7, 10, 25);                           \
  SP_REG3(SPK_B, SPK_FUSED, MF_B_fused, T, DT, 7, 10, 25);                           \
  SP_REG3(SPK_C, SPK_FUSED, MF_C_fused, T, DT, 7, 10, 25);                           \
  SP_REG3(SPK_AMK, SPK_FUSED, MF_AMK_fused, T, DT, 7, 10, 25);                       \
  SP_REG3(SPK_BMK, SPK_FUSED, MF_BMK_fused, T, DT, 7, 10, 25);                       \
  SP_REG2(SPK_A, SPK_FUSED, MF_A_fused, T, DT, 9, 6, 13);                            \
  SP_REG2(SPK_B, SPK_FUSED, MF_B_exact, T, DT, 9, 6, 13);                            \
  SP_REG2(SPK_C, SPK_FUSED, MF_C_exact, T, DT, 9, 6, 13);                            \
  SP_REG3(SPK_A, SPK_FUSED, MF_A_fused, T, DT, 15, 10, 25);                          \
  SP_REG3(SPK_B, SPK_FUSED, MF_B_exact, T, DT, 15, 10, 25);                          \
  SP_REG3(SPK_C, SPK_FUSED, MF_C_exact, T, DT, 15, 10, 25);                         \
  SP_REG2(SPK_A, SPK_FUSED, MF4_A_exact, T, DT, 1009, 1014, 1021);                   \
  SP_REG2(SPK_B, SPK_FUSED, MF4_B_exact, T, DT, 1009, 1014, 1021);                   \
  SP_REG2(SPK_C, SPK_FUSED, MF4_C_exact, T, DT, 1009, 1014, 1021);                   \
  SP_REG2(SPK_AMK, SPK_FUSED, MF4_AMK_exact, T, DT, 1009, 1014, 1021);               \
  SP_REG2(SPK_BMK, SPK_FUSED, MF4_BMK_exact, T, DT, 1009, 1014, 1021);

// extra tile shapes of the FP32 fused kernels, for sp_autotune
#define SP_FUSED_VARIANTS3(MODEL, MF)                                                   \
  SP_REG3T(MODEL, SPK_FUSED, MF, float, 0, 7, 10, 25, ::sp::Tiles<float>::D3b);        \
  SP_REG3T(MODEL, SPK_FUSED, MF, float, 0, 7, 10, 25, ::sp::Tiles<float>::D3c);        \
  SP_REG3T(MODEL, SPK_FUSED, MF, float, 0, 7, 10, 25, ::sp::Tiles<float>::D3d);        \
  SP_REG3T(MODEL, SPK_FUSED, MF, float, 0, 7, 10, 25, ::sp::Tiles<float>::D3e);        \
  SP_REG3T(MODEL, SPK_FUSED, MF, float, 0, 7, 10, 25, ::sp::Tiles<float>::D3f);
// temporally blocked shapes (sp_tb2.cuh) of the FP32 2D fused kernels, for
// sp_autotune: the depth is part of the shape
#define SP_FUSED_TB2(MODEL, MF0, MF1)                                                   \
  SP_REG2TB(MODEL, SPK_FUSED, MF0, MF1, float, 0, 5, 6, 13, ::sp::Tiles<float>::T2a);  \
  SP_REG2TB(MODEL, SPK_FUSED, MF0, MF1, float, 0, 5, 6, 13, ::sp::Tiles<float>::T2b);
#define SP_FUSED_VARIANTS2(MODEL, MF0, MF1)                                             \
  SP_REG2T(MODEL, SPK_FUSED, MF0, MF1, float, 0, 5, 6, 13, ::sp::Tiles<float>::D2b);   \
  SP_REG2T(MODEL, SPK_FUSED, MF0, MF1, float, 0, 5, 6, 13, ::sp::Tiles<float>::D2c);

namespace sp {
void register_fused_kernels() {
  SP_FUSED_SET(float, 0)
  SP_FUSED_SET(double, 1)
  // conserved-pattern kernels (register z-queues) for models B and BMK
  SP_REGCH3(SPK_B, MF_B_fused, ::sp::Tiles<float>::C3a);
  SP_REGCH3(SPK_B, MF_B_fused, ::sp::Tiles<float>::C3b);
  SP_REGCH3(SPK_B, MF_B_fused, ::sp::Tiles<float>::C3c);
  SP_REGCH3(SPK_B, MF_B_fused, ::sp::Tiles<float>::C3d);
  SP_REGCH3(SPK_BMK, MF_BMK_fused, ::sp::Tiles<float>::C3a);
  SP_REGCH3(SPK_BMK, MF_BMK_fused, ::sp::Tiles<float>::C3c);
  SP_FUSED_VARIANTS3(SPK_A, MF_A_fused)
  SP_FUSED_VARIANTS3(SPK_B, MF_B_fused)
  SP_FUSED_VARIANTS3(SPK_C, MF_C_fused)
  SP_FUSED_VARIANTS2(SPK_A, MF_A_fused, MF_A_fused)
  SP_FUSED_VARIANTS2(SPK_B, MF_B_fused, MF_B_fused)
  SP_FUSED_VARIANTS2(SPK_ENS_AB, MF_AMK_fused, MF_BMK_fused)
  SP_FUSED_TB2(SPK_A, MF_A_fused, MF_A_fused)
  SP_FUSED_TB2(SPK_B, MF_B_fused, MF_B_fused)
  SP_FUSED_TB2(SPK_C, MF_C_fused, MF_C_fused)
  SP_FUSED_TB2(SPK_AMK, MF_AMK_fused, MF_AMK_fused)
  SP_FUSED_TB2(SPK_BMK, MF_BMK_fused, MF_BMK_fused)
  SP_FUSED_TB2(SPK_ENS_AB, MF_AMK_fused, MF_BMK_fused)
}
}  // namespace sp
